// C-ABI implementation (include/cupbr_c.h).
#include "../../include/cupbr_c.h"
#include "dev_alloc.hpp"
#include "nvtx_range.hpp"

#include <cmath>
#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "batch.hpp"
#include "cache.hpp"
#include "device_scene.hpp"
#include "pathtracer.hpp"
#include "medium.hpp"
#include "methods.hpp"
#include "post.hpp"

using namespace cupbr_b200;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char* where) {
    return fail(CUPBR_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define CUPBR_CHECK_CUDA(call)                                  \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);     \
    } while (0)

HMaterial to_h(const cupbr_material* m) {
    HMaterial h;
    if (!m) return h;
    h.type = m->type;
    std::memcpy(h.albedo_e, &m->albedo_e, 12);
    std::memcpy(h.albedo_d, &m->albedo_d, 12);
    std::memcpy(h.albedo_s, &m->albedo_s, 12);
    h.shininess = m->shininess;
    h.roughness = m->roughness;
    h.eta = m->eta;
    std::memcpy(h.sigma_s, &m->sigma_s, 12);
    std::memcpy(h.sigma_a, &m->sigma_a, 12);
    h.g = m->g;
    h.interface_glass = m->interface_glass;
    return h;
}
void from_h(const HMaterial& h, cupbr_material* m) {
    m->type = h.type;
    std::memcpy(&m->albedo_e, h.albedo_e, 12);
    std::memcpy(&m->albedo_d, h.albedo_d, 12);
    std::memcpy(&m->albedo_s, h.albedo_s, 12);
    m->shininess = h.shininess;
    m->roughness = h.roughness;
    m->eta = h.eta;
    std::memcpy(&m->sigma_s, h.sigma_s, 12);
    std::memcpy(&m->sigma_a, h.sigma_a, 12);
    m->g = h.g;
    m->interface_glass = h.interface_glass;
}

bool valid_material(const cupbr_material* m, std::string& why) {
    if (m && (m->type < 0 || m->type > 5)) { why = "material type out of range"; return false; }
    return true;
}

BvhBuildParams to_params(const cupbr_bvh_params* p) {
    BvhBuildParams b;
    b.top_bfs_levels = 4;
    if (p) {
        if (p->max_leaf_size >= 1 && p->max_leaf_size <= BVH_MAX_LEAF) b.max_leaf = p->max_leaf_size;
        if (p->traversal_cost > 0.0f) b.trav_cost = p->traversal_cost;
        if (p->top_bfs_levels >= 0 && p->top_bfs_levels <= 8) b.top_bfs_levels = p->top_bfs_levels;
        b.device = p->builder != CUPBR_BVH_BUILD_HOST;
    }
    return b;
}

int device_sm_count() {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 1;
    }
    return sms;
}

// Device buffers of the wavefront tracer for n paths.
struct PTBuffers {
    Workspace ws{};
    uint32_t capacity = 0;
    std::vector<void*> bufs;
    ~PTBuffers() { release(); }
    void release() {
        for (void* p : bufs) cudaFree(p);
        bufs.clear();
        ws = Workspace{};
        capacity = 0;
    }
    cudaError_t alloc(void** p, size_t bytes) {
        cudaError_t e = dev_alloc(p, bytes);
        if (e == cudaSuccess) bufs.push_back(*p);
        return e;
    }
    cudaError_t ensure(uint32_t n) {
        if (n <= capacity) return cudaSuccess;
        release();
        void* p;
        cudaError_t e;
        if ((e = alloc(&p, sizeof(float4) * n)) != cudaSuccess) return e;
        ws.radiance = (float4*)p;
        for (int k = 0; k < 2; ++k) {
            if ((e = alloc(&p, sizeof(float4) * 3 * (size_t)n)) != cudaSuccess) return e;
            ws.rays[k] = (float4*)p;
        }
        if ((e = alloc(&p, sizeof(float2) * n)) != cudaSuccess) return e;
        ws.hits = (float2*)p;
        if ((e = alloc(&p, sizeof(float4) * 3 * (size_t)n)) != cudaSuccess) return e;
        ws.shadow = (float4*)p;
        if ((e = alloc(&p, sizeof(uint32_t) * CTR_TOTAL)) != cudaSuccess) return e;
        ws.ctr = (uint32_t*)p;
        if ((e = alloc(&p, sizeof(uint32_t) * ERR_TOTAL)) != cudaSuccess) return e;
        ws.err = (uint32_t*)p;
        if ((e = cudaMemset(p, 0, sizeof(uint32_t) * ERR_TOTAL)) != cudaSuccess) return e;
        if ((e = alloc(&p, sizeof(uint64_t) * STAT_TOTAL)) != cudaSuccess) return e;
        ws.stats = (uint64_t*)p;
        // no BVH nodes staged in shared memory: with the top 128 nodes
        // staged (16 KB per block) the 1080p heightfield frame measured 3 %
        // slower than with none (the L1 left to the traversal stacks and
        // node loads serves the top of the tree as well)
        ws.smem_nodes = 0;
        ws.trace_blocks_per_sm = pt_occupancy_blocks((int)(ws.smem_nodes * BVH_NODE_BYTES));
        capacity = n;
        return cudaSuccess;
    }
};

// CUDA events of profiled wavefronts: per wavefront [0] start, [1] after the
// camera kernel, `per_depth` stage events per depth, [last] after the
// accumulation (pathtracer.hpp / medium.hpp layouts), summed per stage when
// read.
struct StageEvents {
    struct Frame {
        std::vector<cudaEvent_t> ev;
        uint32_t per_depth;
    };
    std::vector<cudaEvent_t> pool;  // free events
    std::vector<Frame> frames;      // recorded, not yet read
    ~StageEvents() {
        for (auto& f : frames)
            for (cudaEvent_t e : f.ev) cudaEventDestroy(e);
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
    }
    // Creates events up front so that profiled renders create none inside a
    // timed region (event creation is a host driver call that can stall).
    cudaError_t reserve(size_t n) {
        while (pool.size() < n) {
            cudaEvent_t e;
            cudaError_t err = cudaEventCreate(&e);
            if (err != cudaSuccess) return err;
            pool.push_back(e);
        }
        return cudaSuccess;
    }
    cudaError_t take(uint32_t n, std::vector<cudaEvent_t>& out) {
        out.clear();
        while (out.size() < n) {
            if (!pool.empty()) {
                out.push_back(pool.back());
                pool.pop_back();
                continue;
            }
            cudaEvent_t e;
            cudaError_t err = cudaEventCreate(&e);
            if (err != cudaSuccess) return err;
            out.push_back(e);
        }
        return cudaSuccess;
    }
    // ms[0] camera, ms[1 .. per_depth] the per-depth stages, ms[per_depth + 1]
    // accumulation (ms holds per_depth + 2 floats); launches = depth steps.
    cudaError_t read(float* ms, uint32_t per_depth, uint32_t* n_frames, uint32_t* launches) {
        for (uint32_t k = 0; k < per_depth + 2; ++k) ms[k] = 0.0f;
        uint32_t nlaunch = 0, nframes = 0;
        cudaError_t e;
        for (auto& f : frames) {
            if (f.per_depth != per_depth) continue;
            if ((e = cudaEventSynchronize(f.ev.back())) != cudaSuccess) return e;
            const uint32_t depth = (uint32_t)(f.ev.size() - 3) / per_depth;
            float t;
            if ((e = cudaEventElapsedTime(&t, f.ev[0], f.ev[1])) != cudaSuccess) return e;
            ms[0] += t;
            for (uint32_t d = 0; d < depth; ++d)
                for (uint32_t k = 0; k < per_depth; ++k) {
                    const uint32_t i = 1 + per_depth * d + k;
                    if ((e = cudaEventElapsedTime(&t, f.ev[i], f.ev[i + 1])) != cudaSuccess) return e;
                    ms[1 + k] += t;
                }
            const uint32_t i = 1 + per_depth * depth;
            if ((e = cudaEventElapsedTime(&t, f.ev[i], f.ev[i + 1])) != cudaSuccess) return e;
            ms[per_depth + 1] += t;
            nlaunch += depth;
            ++nframes;
        }
        if (n_frames) *n_frames = nframes;
        if (launches) *launches = nlaunch;
        for (auto& f : frames) pool.insert(pool.end(), f.ev.begin(), f.ev.end());
        frames.clear();
        return cudaSuccess;
    }
};

}  // namespace

struct cupbr_scene_s {
    GpuScene g;
    PTBuffers pt;  // workspace for cupbr_pathtracing
};

struct cupbr_renderer_s {
    int32_t method = CUPBR_RAYTRACER;
    uint32_t w = 0, h = 0;
    cupbr_scene_s* scene = nullptr;
    uint32_t frame = 0, max_depth = 5;
    bool rr = false;
    uint32_t estimator = CUPBR_ESTIMATOR_REFERENCE;
    bool size_set = false;
    bool instrumented = false;
    float* hdr = nullptr;
    std::vector<float*> aux;  // gradient-domain buffers (allocated on first use)
    uint64_t* gd_valid = nullptr;  // gradient-domain base-path vertex masks, one per interior pixel and frame
    size_t gd_valid_n = 0;
    PTBuffers pt;
    cudaStream_t stream = nullptr;
    uint64_t last_rays[2] = {0, 0};
    uint32_t batch_paths = 1u << 25;  // paths per wavefront when several frames are rendered at once
    // per-path tail kernel below this queue size (0: off); unless set, 2^17
    // on one stream and 2^16 pipelined, where the other stream's wavefront
    // fills the SMs that a sparse queue leaves idle
    uint32_t tail_paths = 0;
    bool tail_set = false;
    uint32_t tail() const { return tail_set ? tail_paths : (pipelined ? 0u : 1u << 17); }
    // rays of the last wavefront frame: closest-hit and shadow queue sizes
    cudaError_t read_wavefront_rays() {
        uint32_t c[CTR_TOTAL];
        cudaError_t e = cudaMemcpyAsync(c, pt.ws.ctr, sizeof c, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        last_rays[0] = last_rays[1] = 0;
        for (uint32_t d = 0; d < max_depth; ++d) {
            last_rays[0] += c[CTR_RAYS + d];
            last_rays[1] += c[CTR_SHADOW + d];
        }
        return cudaSuccess;
    }
    // ray counts of an instrumented GRADIENTDOMAIN frame (device counters)
    cudaError_t read_method_rays() {
        uint64_t c[STAT_TOTAL];
        cudaError_t e = cudaMemcpyAsync(c, pt.ws.stats, sizeof c, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        last_rays[0] = c[STAT_EXT_RAYS];
        last_rays[1] = c[STAT_SH_RAYS];
        return cudaSuccess;
    }
    bool profiling = false;
    StageEvents events;
    // pipelined PATHTRACER frames: slot k traces on its own stream and
    // workspace; the running mean is folded on the renderer's stream.
    // render() cycles through PIPE_SLOTS slots (single frames leave the GPU
    // part-empty in their late depths, which the other slots' frames fill);
    // render_frames() alternates its large wavefronts between the first two
    static constexpr int PIPE_SLOTS = 4;
    bool pipelined = false;
    uint32_t pipe_next = 0;
    PTBuffers pipe_pt[PIPE_SLOTS];
    uint64_t* pipe_valid[PIPE_SLOTS] = {};  // GRADIENTDOMAIN: the slots' base-path vertex masks
    size_t pipe_valid_n[PIPE_SLOTS] = {};
    cudaStream_t pipe_stream[PIPE_SLOTS] = {};
    cudaEvent_t pipe_traced[PIPE_SLOTS] = {}, pipe_folded[PIPE_SLOTS] = {};
    cudaEvent_t pipe_start = nullptr;  // render_frames: the caller's stream when the call began
    cudaError_t pipe_init() {
        cudaError_t e;
        if (!pipe_start && (e = cudaEventCreateWithFlags(&pipe_start, cudaEventDisableTiming)) != cudaSuccess) return e;
        for (int k = 0; k < PIPE_SLOTS; ++k) {
            // default flags: synchronous copies on the legacy stream (scene
            // edits) still wait for frames in flight here
            if (!pipe_stream[k] && (e = cudaStreamCreate(&pipe_stream[k])) != cudaSuccess) return e;
            if (!pipe_traced[k] && (e = cudaEventCreateWithFlags(&pipe_traced[k], cudaEventDisableTiming)) != cudaSuccess)
                return e;
            if (!pipe_folded[k] && (e = cudaEventCreateWithFlags(&pipe_folded[k], cudaEventDisableTiming)) != cudaSuccess)
                return e;
        }
        return cudaSuccess;
    }
    // render_frames through the batch's persistent kernel (one view): its
    // scene record, view, work items and counter
    bool persistent = false;
    DeviceScene* pk_scene = nullptr;
    BatchView* pk_view = nullptr;
    BatchItem* pk_items = nullptr;
    uint32_t* pk_counter = nullptr;  // [0] item counter, [1] stack overflows
    uint32_t pk_items_n = 0, pk_w = 0, pk_h = 0;
    const cupbr_scene_s* pk_for = nullptr;
    uint64_t pk_gen = 0;
    void pk_release() {
        if (pk_scene) cudaFree(pk_scene);
        if (pk_view) cudaFree(pk_view);
        if (pk_items) cudaFree(pk_items);
        if (pk_counter) cudaFree(pk_counter);
        pk_scene = nullptr;
        pk_view = nullptr;
        pk_items = nullptr;
        pk_counter = nullptr;
        pk_items_n = pk_w = pk_h = 0;
        pk_for = nullptr;
    }
    // frames [frame, frame + n) of one view through the persistent kernel
    // (the same images as the wavefront, bit for bit)
    cudaError_t render_persistent(const cupbr_camera* c, uint32_t n);
    ~cupbr_renderer_s() {
        pk_release();
        for (int k = 0; k < PIPE_SLOTS; ++k) {
            if (pipe_stream[k]) cudaStreamSynchronize(pipe_stream[k]);
            if (pipe_valid[k]) cudaFree(pipe_valid[k]);
            if (pipe_traced[k]) cudaEventDestroy(pipe_traced[k]);
            if (pipe_folded[k]) cudaEventDestroy(pipe_folded[k]);
            if (pipe_stream[k]) cudaStreamDestroy(pipe_stream[k]);
        }
        if (pipe_start) cudaEventDestroy(pipe_start);
        if (hdr) cudaFree(hdr);
        for (float* p : aux) cudaFree(p);
        if (gd_valid) cudaFree(gd_valid);
    }
};

struct cupbr_tonemapper_s {
    int32_t type = CUPBR_REINHARD;
    float exposure = 1.0f;
    const float* hdr = nullptr;
    uint32_t w = 0, h = 0;
    uint8_t* rgba = nullptr;
    cudaStream_t stream = nullptr;
    ~cupbr_tonemapper_s() { if (rgba) cudaFree(rgba); }
};

struct cupbr_postprocessor_s {
    const float* hdr = nullptr;
    uint32_t w = 0, h = 0;
    float* out = nullptr;
    float* half = nullptr;
    cudaStream_t stream = nullptr;
    ~cupbr_postprocessor_s() {
        if (out) cudaFree(out);
        if (half) cudaFree(half);
    }
};

extern "C" {

const char* cupbr_last_error(void) { return g_last_error.c_str(); }
const char* cupbr_version(void) { return "cupbr-b200 0.1 (sm_100a)"; }

int cupbr_material_default(cupbr_material* out) {
    if (!out) return fail(CUPBR_ERR_ARG, "null output");
    from_h(HMaterial(), out);
    return CUPBR_OK;
}

int cupbr_camera_default(uint32_t width, uint32_t height, cupbr_camera* out) {
    if (!out || width == 0 || height == 0) return fail(CUPBR_ERR_ARG, "camera needs a non-zero size");
    const float aspect = static_cast<float>(width) / static_cast<float>(height);  // Camera.cpp:8
    *out = cupbr_camera{{0, 0, 0}, {aspect, 0, 0}, {0, 1, 0}, {0, 0, 1}, aspect, 0};
    return CUPBR_OK;
}

// ------------------------------------------------------------- scene ---
int cupbr_scene_create(cupbr_scene_t* out) {
    if (!out) return fail(CUPBR_ERR_ARG, "null output");
    *out = new cupbr_scene_s();
    return CUPBR_OK;
}

int cupbr_scene_load_xml_ex(const char* path, const cupbr_bvh_params* params, cupbr_scene_t* out) {
    if (!path || !out) return fail(CUPBR_ERR_ARG, "null argument");
    std::unique_ptr<cupbr_scene_s> s(new cupbr_scene_s());
    std::string err;
    if (!load_scene_xml(path, s->g.host, err)) return fail(CUPBR_ERR_IO, err);
    if (!commit_scene(s->g, to_params(params), err)) return fail(CUPBR_ERR_CUDA, err);
    *out = s.release();
    return CUPBR_OK;
}
int cupbr_scene_load_xml(const char* path, cupbr_scene_t* out) { return cupbr_scene_load_xml_ex(path, nullptr, out); }
int cupbr_scene_parse_xml(const char* path, cupbr_scene_t* out) {
    if (!path || !out) return fail(CUPBR_ERR_ARG, "null argument");
    std::unique_ptr<cupbr_scene_s> s(new cupbr_scene_s());
    std::string err;
    if (!load_scene_xml(path, s->g.host, err)) return fail(CUPBR_ERR_IO, err);
    *out = s.release();
    return CUPBR_OK;
}

#define SCENE_MUTABLE(s)                                                                  \
    do {                                                                                  \
        if (!(s)) return fail(CUPBR_ERR_ARG, "null scene");                               \
        if ((s)->g.committed) return fail(CUPBR_ERR_STATE, "scene already committed");    \
    } while (0)

int cupbr_scene_add_sphere(cupbr_scene_t s, cupbr_vec3 position, float radius, const cupbr_material* m, uint32_t* id) {
    SCENE_MUTABLE(s);
    std::string why;
    if (!valid_material(m, why)) return fail(CUPBR_ERR_ARG, why);
    uint32_t i = s->g.host.add_sphere(&position.x, radius, to_h(m));
    if (id) *id = i;
    return CUPBR_OK;
}
int cupbr_scene_add_plane(cupbr_scene_t s, cupbr_vec3 position, cupbr_vec3 normal, const cupbr_material* m, uint32_t* id) {
    SCENE_MUTABLE(s);
    std::string why;
    if (!valid_material(m, why)) return fail(CUPBR_ERR_ARG, why);
    uint32_t i = s->g.host.add_plane(&position.x, &normal.x, to_h(m));
    if (id) *id = i;
    return CUPBR_OK;
}
int cupbr_scene_add_quad(cupbr_scene_t s, cupbr_vec3 position, cupbr_vec3 normal, cupbr_vec3 e1, cupbr_vec3 e2,
                         const cupbr_material* m, uint32_t* id) {
    SCENE_MUTABLE(s);
    std::string why;
    if (!valid_material(m, why)) return fail(CUPBR_ERR_ARG, why);
    uint32_t i = s->g.host.add_quad(&position.x, &normal.x, &e1.x, &e2.x, to_h(m));
    if (id) *id = i;
    return CUPBR_OK;
}
int cupbr_scene_add_triangle(cupbr_scene_t s, cupbr_vec3 v1, cupbr_vec3 v2, cupbr_vec3 v3, const cupbr_material* m,
                             uint32_t* id) {
    SCENE_MUTABLE(s);
    std::string why;
    if (!valid_material(m, why)) return fail(CUPBR_ERR_ARG, why);
    uint32_t i = s->g.host.add_triangle(&v1.x, &v2.x, &v3.x, to_h(m));
    if (id) *id = i;
    return CUPBR_OK;
}
int cupbr_scene_add_mesh(cupbr_scene_t s, const float* vertices, uint32_t nv, const uint32_t* indices, uint32_t nt,
                         cupbr_vec3 position, cupbr_vec3 scale, const cupbr_material* m, uint32_t* id) {
    SCENE_MUTABLE(s);
    std::string why;
    if (!valid_material(m, why)) return fail(CUPBR_ERR_ARG, why);
    if ((nv && !vertices) || (nt && !indices)) return fail(CUPBR_ERR_ARG, "null mesh arrays");
    for (uint64_t k = 0; k < 3ull * nt; ++k)
        if (indices[k] >= nv) return fail(CUPBR_ERR_ARG, "mesh index out of range");
    for (uint64_t k = 0; k < 3ull * nv; ++k)
        if (!std::isfinite(vertices[k])) return fail(CUPBR_ERR_ARG, "non-finite mesh vertex");
    uint32_t i = s->g.host.add_mesh(vertices, nv, indices, nt, &position.x, &scale.x, to_h(m));
    if (id) *id = i;
    return CUPBR_OK;
}
int cupbr_scene_add_mesh_obj(cupbr_scene_t s, const char* path, cupbr_vec3 position, cupbr_vec3 scale,
                             const cupbr_material* m, uint32_t* id) {
    SCENE_MUTABLE(s);
    if (!path) return fail(CUPBR_ERR_ARG, "null path");
    std::vector<float> v;
    std::vector<uint32_t> idx;
    std::string err;
    if (!load_obj(path, v, idx, err)) return fail(CUPBR_ERR_IO, err);
    return cupbr_scene_add_mesh(s, v.data(), (uint32_t)(v.size() / 3), idx.data(), (uint32_t)(idx.size() / 3), position,
                                scale, m, id);
}
int cupbr_scene_add_light(cupbr_scene_t s, const cupbr_light* l) {
    SCENE_MUTABLE(s);
    if (!l || (l->type != CUPBR_POINT && l->type != CUPBR_AREA)) return fail(CUPBR_ERR_ARG, "bad light");
    HLight h;
    h.type = l->type;
    std::memcpy(h.position, &l->position, 12);
    std::memcpy(h.intensity, &l->intensity, 12);
    std::memcpy(h.radiance, &l->radiance, 12);
    std::memcpy(h.he1, &l->half_extend1, 12);
    std::memcpy(h.he2, &l->half_extend2, 12);
    s->g.host.lights.push_back(h);
    return CUPBR_OK;
}
int cupbr_scene_set_volume(cupbr_scene_t s, cupbr_vec3 sigma_s, cupbr_vec3 sigma_a, float g) {
    SCENE_MUTABLE(s);
    std::memcpy(s->g.host.vol_sigma_s, &sigma_s, 12);
    std::memcpy(s->g.host.vol_sigma_a, &sigma_a, 12);
    s->g.host.vol_g = g;
    return CUPBR_OK;
}
int cupbr_scene_set_environment(cupbr_scene_t s, const float* rgb, uint32_t w, uint32_t h) {
    SCENE_MUTABLE(s);
    if (!rgb || w == 0 || h == 0) return fail(CUPBR_ERR_ARG, "empty environment map");
    s->g.host.env.assign(rgb, rgb + (size_t)w * h * 3);
    s->g.host.env_w = w;
    s->g.host.env_h = h;
    return CUPBR_OK;
}
int cupbr_scene_set_albedo_texture(cupbr_scene_t s, const float* rgb, uint32_t w, uint32_t h) {
    SCENE_MUTABLE(s);
    if (!rgb || w == 0 || h == 0) return fail(CUPBR_ERR_ARG, "empty albedo texture");
    if ((uint64_t)w * h > (1ull << 28)) return fail(CUPBR_ERR_ARG, "albedo texture above 2^28 texels");
    const size_t n = (size_t)w * h * 3;
    for (size_t i = 0; i < n; ++i)
        if (!(rgb[i] >= 0.0f) || !std::isfinite(rgb[i])) return fail(CUPBR_ERR_ARG, "albedo texel not finite and >= 0");
    s->g.host.tex.assign(rgb, rgb + n);
    s->g.host.tex_w = w;
    s->g.host.tex_h = h;
    return CUPBR_OK;
}
int cupbr_scene_set_object_texture(cupbr_scene_t s, uint32_t object, cupbr_vec3 origin, cupbr_vec3 u_axis,
                                   cupbr_vec3 v_axis) {
    SCENE_MUTABLE(s);
    if (object >= s->g.host.objects.size()) return fail(CUPBR_ERR_ARG, "object index out of range");
    const float uu = u_axis.x * u_axis.x + u_axis.y * u_axis.y + u_axis.z * u_axis.z;
    const float vv = v_axis.x * v_axis.x + v_axis.y * v_axis.y + v_axis.z * v_axis.z;
    if (!(uu > 0.0f) || !(vv > 0.0f) || !std::isfinite(uu) || !std::isfinite(vv))
        return fail(CUPBR_ERR_ARG, "texture axes must be finite and non-zero");
    HObject& ob = s->g.host.objects[object];
    ob.textured = true;
    const float o3[3] = {origin.x, origin.y, origin.z}, u3[3] = {u_axis.x, u_axis.y, u_axis.z},
                v3[3] = {v_axis.x, v_axis.y, v_axis.z};
    for (int k = 0; k < 3; ++k) {
        ob.tex_origin[k] = o3[k];
        ob.tex_u[k] = u3[k];
        ob.tex_v[k] = v3[k];
    }
    return CUPBR_OK;
}
int cupbr_scene_get_albedo_texture(cupbr_scene_t s, float** device_texels, uint32_t* w, uint32_t* h) {
    if (!s || !device_texels) return fail(CUPBR_ERR_ARG, "null argument");
    if (!s->g.committed) return fail(CUPBR_ERR_STATE, "scene not committed");
    *device_texels = reinterpret_cast<float*>(s->g.dev.tex);
    if (w) *w = s->g.dev.tex_w;
    if (h) *h = s->g.dev.tex_h;
    return CUPBR_OK;
}
int cupbr_scene_load_environment(cupbr_scene_t s, const char* path) {
    SCENE_MUTABLE(s);
    if (!path) return fail(CUPBR_ERR_ARG, "null path");
    std::string err, p(path);
    bool ok = (p.size() > 4 && p.compare(p.size() - 4, 4, ".pfm") == 0)
                  ? read_pfm(p, s->g.host.env, s->g.host.env_w, s->g.host.env_h, err)
                  : load_hdr_image(p, s->g.host.env, s->g.host.env_w, s->g.host.env_h, err);
    return ok ? CUPBR_OK : fail(CUPBR_ERR_IO, err);
}
int cupbr_scene_commit(cupbr_scene_t s, const cupbr_bvh_params* params) {
    NvtxRange nvtx_("cupbr_scene_commit");
    SCENE_MUTABLE(s);
    std::string err;
    if (!commit_scene(s->g, to_params(params), err)) return fail(CUPBR_ERR_CUDA, err);
    return CUPBR_OK;
}
int cupbr_scene_destroy(cupbr_scene_t s) {
    delete s;
    return CUPBR_OK;
}
int cupbr_scene_get_info(cupbr_scene_t s, cupbr_scene_info* o) {
    if (!s || !o) return fail(CUPBR_ERR_ARG, "null argument");
    std::memset(o, 0, sizeof *o);
    const HostScene& h = s->g.host;
    o->objects = (uint32_t)h.objects.size();
    o->lights = (uint32_t)h.lights.size();
    for (const HObject& ob : h.objects) {
        if (ob.type == GEO_MESH || ob.type == GEO_TRIANGLE) o->triangles += ob.tri_count;
        else if (ob.type == GEO_SPHERE) o->spheres++;
        else if (ob.type == GEO_QUAD) o->quads++;
        else o->planes++;
    }
    o->bvh_nodes = s->g.dev.n_nodes;
    o->bvh_leaves = s->g.bvh.stats.leaves;
    o->bvh_depth = s->g.bvh.stats.max_depth;
    o->bvh_sah_cost = s->g.bvh.stats.sah_cost;
    o->device_bytes = s->g.device_bytes;
    o->env_width = h.env_w;
    o->env_height = h.env_h;
    o->committed = s->g.committed ? 1 : 0;
    o->bvh_builder = s->g.bvh_device ? CUPBR_BVH_BUILD_DEVICE : CUPBR_BVH_BUILD_HOST;
    o->bvh_build_ms = s->g.bvh_ms;
    o->commit_ms = s->g.commit_ms;
    return CUPBR_OK;
}
int cupbr_scene_get_object(cupbr_scene_t s, uint32_t index, cupbr_object_desc* o) {
    if (!s || !o) return fail(CUPBR_ERR_ARG, "null argument");
    if (index >= s->g.host.objects.size()) return fail(CUPBR_ERR_ARG, "object index out of range");
    const HObject& ob = s->g.host.objects[index];
    o->type = ob.type;
    from_h(ob.mat, &o->material);
    std::memcpy(&o->p0, ob.p0, 12);
    std::memcpy(&o->p1, ob.p1, 12);
    std::memcpy(&o->p2, ob.p2, 12);
    std::memcpy(&o->p3, ob.p3, 12);
    o->radius = ob.radius;
    o->triangle_begin = ob.tri_begin;
    o->triangle_count = ob.tri_count;
    o->finite_box = ob.finite_box ? 1 : 0;
    std::memcpy(&o->box_lo, ob.box_lo, 12);
    std::memcpy(&o->box_hi, ob.box_hi, 12);
    return CUPBR_OK;
}
int cupbr_scene_get_triangles(cupbr_scene_t s, uint32_t index, float* out, uint32_t cap) {
    if (!s || !out) return fail(CUPBR_ERR_ARG, "null argument");
    if (index >= s->g.host.objects.size()) return fail(CUPBR_ERR_ARG, "object index out of range");
    const HObject& ob = s->g.host.objects[index];
    if (cap < ob.tri_count) return fail(CUPBR_ERR_ARG, "capacity too small");
    std::memcpy(out, &s->g.host.tri_verts[9 * (size_t)ob.tri_begin], sizeof(float) * 9 * (size_t)ob.tri_count);
    return CUPBR_OK;
}
int cupbr_scene_get_bvh(cupbr_scene_t s, float* out, uint32_t cap, uint32_t* n_nodes) {
    if (!s || !n_nodes) return fail(CUPBR_ERR_ARG, "null argument");
    if (!s->g.committed) return fail(CUPBR_ERR_STATE, "scene not committed");
    *n_nodes = s->g.dev.n_nodes;
    if (!out) return CUPBR_OK;
    if (cap < s->g.dev.n_nodes) return fail(CUPBR_ERR_ARG, "capacity too small");
    CUPBR_CHECK_CUDA(cudaMemcpy(out, s->g.dev.nodes, (size_t)s->g.dev.n_nodes * BVH_NODE_BYTES, cudaMemcpyDeviceToHost));
    return CUPBR_OK;
}
int cupbr_scene_get_key_slots(cupbr_scene_t s, uint32_t* out, uint32_t cap, uint32_t* n_keys) {
    if (!s || !n_keys) return fail(CUPBR_ERR_ARG, "null argument");
    if (!s->g.committed) return fail(CUPBR_ERR_STATE, "scene not committed");
    const uint32_t n = (uint32_t)s->g.key_obj.size();
    *n_keys = n;
    if (!out || n == 0) return CUPBR_OK;
    if (cap < n) return fail(CUPBR_ERR_ARG, "capacity too small");
    CUPBR_CHECK_CUDA(cudaMemcpy(out, s->g.dev.key_slot, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return CUPBR_OK;
}
int cupbr_scene_get_camera(cupbr_scene_t s, uint32_t width, uint32_t height, cupbr_camera* out) {
    if (!s || !out) return fail(CUPBR_ERR_ARG, "null argument");
    if (int rc = cupbr_camera_default(width, height, out)) return rc;
    const HCamera& c = s->g.host.camera;
    if (!c.set) return CUPBR_OK;
    // Camera.cpp:82-88, in float as the reference computes it
    const float a = out->aspect_ratio;
    const float zx = std::cos(c.yaw) * std::cos(c.pitch), zy = std::sin(c.pitch), zz = std::sin(c.yaw) * std::cos(c.pitch);
    const float hx = zz, hz = -zx;
    const float hn = std::sqrt(hx * hx + hz * hz);
    const float xx = a * (hx / hn), xy = a * (0.0f / hn), xz = a * (hz / hn);
    out->position = {c.position[0], c.position[1], c.position[2]};
    out->z_axis = {zx, zy, zz};
    out->x_axis = {xx, xy, xz};
    out->y_axis = {(zy * xz - zz * xy) / a, (zz * xx - zx * xz) / a, (zx * xy - zy * xx) / a};
    return CUPBR_OK;
}
int cupbr_scene_set_camera(cupbr_scene_t s, cupbr_vec3 position, float yaw, float pitch) {
    if (!s) return fail(CUPBR_ERR_ARG, "null scene");
    HCamera& c = s->g.host.camera;
    c.set = true;
    c.position[0] = position.x;
    c.position[1] = position.y;
    c.position[2] = position.z;
    c.yaw = yaw;
    c.pitch = std::max(-3.14159f / 2.0f, std::min(3.14159f / 2.0f, pitch));
    return CUPBR_OK;
}
int cupbr_scene_get_light(cupbr_scene_t s, uint32_t index, cupbr_light* o) {
    if (!s || !o) return fail(CUPBR_ERR_ARG, "null argument");
    if (index >= s->g.host.lights.size()) return fail(CUPBR_ERR_ARG, "light index out of range");
    const HLight& l = s->g.host.lights[index];
    o->type = l.type;
    std::memcpy(&o->position, l.position, 12);
    std::memcpy(&o->intensity, l.intensity, 12);
    std::memcpy(&o->radiance, l.radiance, 12);
    std::memcpy(&o->half_extend1, l.he1, 12);
    std::memcpy(&o->half_extend2, l.he2, 12);
    return CUPBR_OK;
}

static int trace_common(cupbr_scene_t s, uint32_t n, const float* o, const float* d, const float* dist, float* depth,
                        int32_t* obj, int32_t* tri, int32_t* vis) {
    if (!s || !o || !d) return fail(CUPBR_ERR_ARG, "null argument");
    if (!s->g.committed) return fail(CUPBR_ERR_STATE, "scene not committed");
    if (n == 0) return CUPBR_OK;
    const size_t v3b = sizeof(float) * 3 * (size_t)n;
    void *dO, *dD, *dDist = nullptr, *dT, *dP, *dK, *dV, *dE;
    CUPBR_CHECK_CUDA(dev_alloc(&dO, v3b));
    CUPBR_CHECK_CUDA(dev_alloc(&dD, v3b));
    CUPBR_CHECK_CUDA(dev_alloc(&dT, sizeof(float) * n));
    CUPBR_CHECK_CUDA(dev_alloc(&dP, sizeof(int32_t) * n));
    CUPBR_CHECK_CUDA(dev_alloc(&dK, sizeof(uint32_t) * n));
    CUPBR_CHECK_CUDA(dev_alloc(&dV, sizeof(int32_t) * n));
    CUPBR_CHECK_CUDA(dev_alloc(&dE, sizeof(uint32_t)));
    CUPBR_CHECK_CUDA(cudaMemset(dE, 0, sizeof(uint32_t)));
    CUPBR_CHECK_CUDA(cudaMemcpy(dO, o, v3b, cudaMemcpyHostToDevice));
    CUPBR_CHECK_CUDA(cudaMemcpy(dD, d, v3b, cudaMemcpyHostToDevice));
    if (dist) {
        CUPBR_CHECK_CUDA(dev_alloc(&dDist, sizeof(float) * n));
        CUPBR_CHECK_CUDA(cudaMemcpy(dDist, dist, sizeof(float) * n, cudaMemcpyHostToDevice));
    }
    CUPBR_CHECK_CUDA(launch_trace_rays(s->g.dev, n, (const float*)dO, (const float*)dD, (const float*)dDist, (float*)dT,
                                       (int32_t*)dP, (uint32_t*)dK, (int32_t*)dV, (uint32_t*)dE, nullptr));
    CUPBR_CHECK_CUDA(cudaDeviceSynchronize());
    uint32_t errc = 0;
    CUPBR_CHECK_CUDA(cudaMemcpy(&errc, dE, 4, cudaMemcpyDeviceToHost));
    if (dist) {
        CUPBR_CHECK_CUDA(cudaMemcpy(vis, dV, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    } else {
        std::vector<int32_t> prim(n);
        std::vector<uint32_t> key(n);
        CUPBR_CHECK_CUDA(cudaMemcpy(depth, dT, sizeof(float) * n, cudaMemcpyDeviceToHost));
        CUPBR_CHECK_CUDA(cudaMemcpy(prim.data(), dP, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        CUPBR_CHECK_CUDA(cudaMemcpy(key.data(), dK, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < n; ++i) {
            if (prim[i] == HIT_NONE) {
                if (obj) obj[i] = -1;
                if (tri) tri[i] = -1;
                continue;
            }
            int32_t ob = s->g.key_obj[key[i]];
            if (obj) obj[i] = ob;
            int gt = s->g.host.objects[ob].type;
            if (tri) tri[i] = (gt == GEO_MESH || gt == GEO_TRIANGLE) ? (int32_t)(key[i] - s->g.key_base[ob]) : -1;
        }
    }
    for (void* p : {dO, dD, dDist, dT, dP, dK, dV, dE})
        if (p) cudaFree(p);
    if (errc) return fail(CUPBR_ERR_STATE, "traversal stack overflow on " + std::to_string(errc) + " rays");
    return CUPBR_OK;
}
int cupbr_scene_trace(cupbr_scene_t s, uint32_t n, const float* o, const float* d, float* depth, int32_t* obj,
                      int32_t* tri) {
    if (!depth) return fail(CUPBR_ERR_ARG, "null depth output");
    return trace_common(s, n, o, d, nullptr, depth, obj, tri, nullptr);
}
int cupbr_scene_visible(cupbr_scene_t s, uint32_t n, const float* o, const float* d, const float* dist, int32_t* vis) {
    if (!dist || !vis) return fail(CUPBR_ERR_ARG, "null argument");
    return trace_common(s, n, o, d, dist, nullptr, nullptr, nullptr, vis);
}

// Interaction::pickMouse, MousePicker.cu:8-35 / :55-72: the un-jittered camera
// ray of pixel (x, y) (Tracing::launchRay, TracingDetail.h:32-44), formed
// here in the device's float operation order and traced on the device.
int cupbr_scene_pick(cupbr_scene_t s, const cupbr_camera* cam, uint32_t x, uint32_t y, uint32_t width,
                     uint32_t height, cupbr_material* out_material, int32_t* out_scene_index) {
    if (!s || !cam || !out_material || !out_scene_index) return fail(CUPBR_ERR_ARG, "null argument");
    if (width == 0 || height == 0 || x >= width || y >= height) return fail(CUPBR_ERR_ARG, "pixel outside the image");
    const float rx = 2.0f * (static_cast<float>(x) / static_cast<float>(width) - 0.5f);
    const float ry = 2.0f * (static_cast<float>(y) / static_cast<float>(height) - 0.5f);
    const cupbr_vec3 p = cam->position, ax = cam->x_axis, ay = cam->y_axis, az = cam->z_axis;
    // position + zAxis + rx * xAxis + ry * yAxis, then minus position
    const float wx = ((p.x + az.x) + rx * ax.x) + ry * ay.x;
    const float wy = ((p.y + az.y) + rx * ax.y) + ry * ay.y;
    const float wz = ((p.z + az.z) + rx * ax.z) + ry * ay.z;
    const float o[3] = {p.x, p.y, p.z};
    const float d[3] = {wx - p.x, wy - p.y, wz - p.z};
    float depth = 0.0f;
    int32_t obj = -1, tri = -1;
    if (int rc = trace_common(s, 1, o, d, nullptr, &depth, &obj, &tri, nullptr)) return rc;
    if (obj < 0) return CUPBR_OK;  // no hit: outputs untouched, as in the reference
    from_h(s->g.host.objects[obj].mat, out_material);
    *out_scene_index = obj;
    return CUPBR_OK;
}

// Interaction::updateMaterial, MousePicker.cu:37-50 / :74-81: every field
// but the glass interface flag, which the reference does not copy either.
int cupbr_scene_update_material(cupbr_scene_t s, int32_t scene_index, const cupbr_material* m) {
    if (!s || !m) return fail(CUPBR_ERR_ARG, "null argument");
    if (scene_index < 0 || (size_t)scene_index >= s->g.host.objects.size())
        return fail(CUPBR_ERR_ARG, "scene index out of range");
    std::string why;
    if (!valid_material(m, why)) return fail(CUPBR_ERR_ARG, why);
    HMaterial& hm = s->g.host.objects[scene_index].mat;
    const bool glass_interface = hm.interface_glass;
    hm = to_h(m);
    hm.interface_glass = glass_interface;
    if (s->g.committed) {
        const DMaterial dm = device_material(hm);
        CUPBR_CHECK_CUDA(cudaMemcpy(const_cast<DMaterial*>(s->g.dev.materials) + scene_index, &dm, sizeof dm,
                                    cudaMemcpyHostToDevice));
    }
    return CUPBR_OK;
}

// ----------------------------------------------------------- renderer ---
static PTFrame make_frame(const cupbr_camera* c, uint32_t w, uint32_t h, uint32_t frame, uint32_t depth, bool rr,
                          uint32_t estimator = CUPBR_ESTIMATOR_REFERENCE) {
    PTFrame F;
    F.estimator = estimator;
    F.width = w;
    F.height = h;
    F.pixels = w * h;
    F.frames = 1;
    F.n_paths = w * h;
    F.frame_index = frame;
    F.max_depth = depth;
    F.use_rr = rr ? 1u : 0u;
    F.cam_pos = mk(c->position.x, c->position.y, c->position.z);
    F.cam_x = mk(c->x_axis.x, c->x_axis.y, c->x_axis.z);
    F.cam_y = mk(c->y_axis.x, c->y_axis.y, c->y_axis.z);
    F.cam_z = mk(c->z_axis.x, c->z_axis.y, c->z_axis.z);
    return F;
}

// n PBRendering::gradientdomain frames: their paths in wavefronts of up to
// the batch path budget (whole frames), each frame then folded into the
// running means and reconstructed in order, as n render() calls.
static int render_gdpt(cupbr_renderer_t r, const cupbr_camera* cam, uint32_t n) {
    if (cam->moved) r->frame = 0;
    if (r->max_depth > PT_MAX_DEPTH) return fail(CUPBR_ERR_ARG, "max trace depth above 64");
    if (r->aux.size() < 8) {
        const size_t bytes = sizeof(float) * 3 * (size_t)r->w * r->h;
        while (r->aux.size() < 8) {
            float* p = nullptr;
            CUPBR_CHECK_CUDA(dev_alloc(&p, bytes));
            r->aux.push_back(p);
            CUPBR_CHECK_CUDA(cudaMemsetAsync(p, 0, bytes, r->stream));
        }
    }
    const uint64_t n_int = r->w >= 3 && r->h >= 3 ? (uint64_t)(r->w - 2) * (r->h - 2) : 0ull;
    if (5ull * n_int > 0xFFFFFFFFull) return fail(CUPBR_ERR_ARG, "image too large for GRADIENTDOMAIN");
    if (n == 1 && r->pipelined && !r->profiling && !r->instrumented) {
        // as the path tracer's pipelined render(): the paths traced on slot
        // k, the running means and reconstruction on the renderer's stream
        // in frame order
        const uint32_t k = r->pipe_next % cupbr_renderer_s::PIPE_SLOTS;
        r->pipe_next = (k + 1) % cupbr_renderer_s::PIPE_SLOTS;
        CUPBR_CHECK_CUDA(r->pipe_init());
        CUPBR_CHECK_CUDA(r->pipe_pt[k].ensure((uint32_t)std::max<uint64_t>(1, 5ull * n_int)));
        const size_t nv = std::max<size_t>(1, (size_t)n_int);
        if (r->pipe_valid_n[k] < nv) {
            // the slot's previous frame may still read its masks
            CUPBR_CHECK_CUDA(cudaStreamSynchronize(r->pipe_stream[k]));
            if (r->pipe_valid[k]) cudaFree(r->pipe_valid[k]);
            r->pipe_valid[k] = nullptr;
            r->pipe_valid_n[k] = 0;
            CUPBR_CHECK_CUDA(dev_alloc(&r->pipe_valid[k], sizeof(uint64_t) * nv));
            r->pipe_valid_n[k] = nv;
        }
        PTFrame F = make_frame(cam, r->w, r->h, r->frame, r->max_depth, false);
        const Workspace& W = r->pipe_pt[k].ws;
        CUPBR_CHECK_CUDA(cudaStreamWaitEvent(r->pipe_stream[k], r->pipe_folded[k], 0));
        CUPBR_CHECK_CUDA(gdpt_trace_frames(r->scene->g.dev, F, W, r->pipe_valid[k], r->pipe_stream[k],
                                           device_sm_count(), false));
        CUPBR_CHECK_CUDA(cudaEventRecord(r->pipe_traced[k], r->pipe_stream[k]));
        CUPBR_CHECK_CUDA(cudaStreamWaitEvent(r->stream, r->pipe_traced[k], 0));
        CUPBR_CHECK_CUDA(gdpt_fold_frames(F, W, r->aux.data(), r->hdr, r->stream));
        CUPBR_CHECK_CUDA(cudaEventRecord(r->pipe_folded[k], r->stream));
        ++r->frame;
        return CUPBR_OK;
    }
    // frames per wavefront: one when instrumented (its counts are per frame)
    uint32_t per = 1;
    if (n_int && !r->instrumented)
        per = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(n, r->batch_paths / (5ull * n_int)));
    CUPBR_CHECK_CUDA(r->pt.ensure((uint32_t)std::max<uint64_t>(1, 5ull * n_int * per)));
    const size_t nv = std::max<size_t>(1, (size_t)n_int * per);
    if (r->gd_valid_n < nv) {
        if (r->gd_valid) cudaFree(r->gd_valid);
        r->gd_valid = nullptr;
        r->gd_valid_n = 0;
        CUPBR_CHECK_CUDA(dev_alloc(&r->gd_valid, sizeof(uint64_t) * nv));
        r->gd_valid_n = nv;
    }
    for (uint32_t done = 0; done < n;) {
        const uint32_t k = std::min(per, n - done);
        PTFrame F = make_frame(cam, r->w, r->h, r->frame, r->max_depth, false);
        F.frames = k;
        if (r->instrumented)
            CUPBR_CHECK_CUDA(cudaMemsetAsync(r->pt.ws.stats, 0, sizeof(uint64_t) * STAT_TOTAL, r->stream));
        CUPBR_CHECK_CUDA(gdpt_trace_frames(r->scene->g.dev, F, r->pt.ws, r->gd_valid, r->stream, device_sm_count(),
                                           r->instrumented));
        CUPBR_CHECK_CUDA(gdpt_fold_frames(F, r->pt.ws, r->aux.data(), r->hdr, r->stream));
        if (r->instrumented) CUPBR_CHECK_CUDA(r->read_method_rays());
        r->frame += k;
        done += k;
    }
    return CUPBR_OK;
}

int cupbr_renderer_create(int32_t method, cupbr_renderer_t* out) {
    if (!out) return fail(CUPBR_ERR_ARG, "null output");
    if (method < 0 || method > 5) return fail(CUPBR_ERR_ARG, "unknown rendering method");
    cupbr_renderer_s* r = new cupbr_renderer_s();
    r->method = method;
    *out = r;
    return CUPBR_OK;
}
int cupbr_renderer_destroy(cupbr_renderer_t r) {
    delete r;
    return CUPBR_OK;
}
int cupbr_renderer_set_output_size(cupbr_renderer_t r, uint32_t w, uint32_t h) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    if (w == 0 || h == 0 || (uint64_t)w * h >= (1ull << 30)) return fail(CUPBR_ERR_ARG, "bad output size");
    if (r->hdr) cudaFree(r->hdr);
    for (float* p : r->aux) cudaFree(p);
    r->aux.clear();
    if (r->gd_valid) cudaFree(r->gd_valid);
    r->gd_valid = nullptr;
    r->gd_valid_n = 0;
    r->hdr = nullptr;
    r->pt.release();
    CUPBR_CHECK_CUDA(dev_alloc(&r->hdr, sizeof(float) * 3 * (size_t)w * h));
    CUPBR_CHECK_CUDA(cudaMemset(r->hdr, 0, sizeof(float) * 3 * (size_t)w * h));
    CUPBR_CHECK_CUDA(r->pt.ensure(w * h));
    r->w = w;
    r->h = h;
    r->size_set = true;
    return CUPBR_OK;
}
int cupbr_renderer_register_scene(cupbr_renderer_t r, cupbr_scene_t s) {
    if (!r || !s) return fail(CUPBR_ERR_ARG, "null argument");
    if (!s->g.committed) return fail(CUPBR_ERR_STATE, "scene not committed");
    r->scene = s;
    return CUPBR_OK;
}
int cupbr_renderer_set_method(cupbr_renderer_t r, int32_t method) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    if (method < 0 || method > 5) return fail(CUPBR_ERR_ARG, "unknown rendering method");
    r->method = method;
    r->frame = 0;
    if (r->hdr) CUPBR_CHECK_CUDA(cudaMemsetAsync(r->hdr, 0, sizeof(float) * 3 * (size_t)r->w * r->h, r->stream));
    for (float* p : r->aux) CUPBR_CHECK_CUDA(cudaMemsetAsync(p, 0, sizeof(float) * 3 * (size_t)r->w * r->h, r->stream));
    return CUPBR_OK;
}
int cupbr_renderer_set_estimator(cupbr_renderer_t r, int32_t estimator) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    if (estimator != CUPBR_ESTIMATOR_REFERENCE && estimator != CUPBR_ESTIMATOR_PHYSICAL)
        return fail(CUPBR_ERR_ARG, "unknown estimator");
    r->estimator = (uint32_t)estimator;
    r->frame = 0;
    if (r->hdr) CUPBR_CHECK_CUDA(cudaMemsetAsync(r->hdr, 0, sizeof(float) * 3 * (size_t)r->w * r->h, r->stream));
    return CUPBR_OK;
}
int cupbr_renderer_get_estimator(cupbr_renderer_t r, int32_t* estimator) {
    if (!r || !estimator) return fail(CUPBR_ERR_ARG, "null argument");
    *estimator = (int32_t)r->estimator;
    return CUPBR_OK;
}
int cupbr_renderer_get_method(cupbr_renderer_t r, int32_t* m) {
    if (!r || !m) return fail(CUPBR_ERR_ARG, "null argument");
    *m = r->method;
    return CUPBR_OK;
}
int cupbr_renderer_render(cupbr_renderer_t r, const cupbr_camera* cam) {
    NvtxRange nvtx_("cupbr_renderer_render");
    if (!r || !cam) return fail(CUPBR_ERR_ARG, "null argument");
    if (!r->size_set) return fail(CUPBR_ERR_STATE, "No output size set. Use setOutputSize()");
    if (!r->scene) return fail(CUPBR_ERR_STATE, "No scene registered. Use registerScene()");
    switch (r->method) {
        case CUPBR_PATHTRACER: {
            if (cam->moved) r->frame = 0;  // PBRenderer.cu:174-177
            if (r->max_depth > PT_MAX_DEPTH) return fail(CUPBR_ERR_ARG, "max trace depth above 64");
            PTFrame F = make_frame(cam, r->w, r->h, r->frame, r->max_depth, r->rr, r->estimator);
            if (r->pipelined && !r->profiling && !r->instrumented) {
                // trace on slot k while the previous frame is still folded,
                // tone mapped or read back on the renderer's stream
                const uint32_t k = r->pipe_next % cupbr_renderer_s::PIPE_SLOTS;
                r->pipe_next = (k + 1) % cupbr_renderer_s::PIPE_SLOTS;
                CUPBR_CHECK_CUDA(r->pipe_init());
                CUPBR_CHECK_CUDA(r->pipe_pt[k].ensure(r->w * r->h));
                const Workspace& W = r->pipe_pt[k].ws;
                // the slot's workspace is free once its last frame was folded
                CUPBR_CHECK_CUDA(cudaStreamWaitEvent(r->pipe_stream[k], r->pipe_folded[k], 0));
                CUPBR_CHECK_CUDA(pt_render_frame(r->scene->g.dev, F, W, nullptr, r->pipe_stream[k], device_sm_count(),
                                                 false, nullptr, r->tail()));
                CUPBR_CHECK_CUDA(cudaEventRecord(r->pipe_traced[k], r->pipe_stream[k]));
                CUPBR_CHECK_CUDA(cudaStreamWaitEvent(r->stream, r->pipe_traced[k], 0));
                CUPBR_CHECK_CUDA(pt_launch_accumulate(F, W, r->hdr, r->stream));
                CUPBR_CHECK_CUDA(cudaEventRecord(r->pipe_folded[k], r->stream));
                ++r->frame;
                return CUPBR_OK;
            }
            if (r->instrumented) CUPBR_CHECK_CUDA(cudaMemsetAsync(r->pt.ws.stats, 0, sizeof(uint64_t) * STAT_TOTAL, r->stream));
            std::vector<cudaEvent_t> ev;
            if (r->profiling) CUPBR_CHECK_CUDA(r->events.take(pt_event_count(r->max_depth), ev));
            CUPBR_CHECK_CUDA(pt_render_frame(r->scene->g.dev, F, r->pt.ws, r->hdr, r->stream, device_sm_count(),
                                             r->instrumented, r->profiling ? ev.data() : nullptr, r->tail()));
            if (r->profiling) r->events.frames.push_back({std::move(ev), 3u});
            if (r->instrumented) CUPBR_CHECK_CUDA(r->read_wavefront_rays());
            ++r->frame;
            return CUPBR_OK;
        }
        case CUPBR_VOLUME: {  // PBRenderer.cu:215-228
            if (cam->moved) r->frame = 0;
            if (r->max_depth > PT_MAX_DEPTH) return fail(CUPBR_ERR_ARG, "max trace depth above 64");
            PTFrame F = make_frame(cam, r->w, r->h, r->frame, r->max_depth, r->rr, r->estimator);
            if (r->pipelined && !r->profiling && !r->instrumented) {
                // as the path tracer's pipelined render(): traced on slot k,
                // folded on the renderer's stream in frame order
                const uint32_t k = r->pipe_next % cupbr_renderer_s::PIPE_SLOTS;
                r->pipe_next = (k + 1) % cupbr_renderer_s::PIPE_SLOTS;
                CUPBR_CHECK_CUDA(r->pipe_init());
                CUPBR_CHECK_CUDA(r->pipe_pt[k].ensure(F.n_paths));
                const Workspace& W = r->pipe_pt[k].ws;
                CUPBR_CHECK_CUDA(cudaStreamWaitEvent(r->pipe_stream[k], r->pipe_folded[k], 0));
                CUPBR_CHECK_CUDA(volume_render_frame(r->scene->g.dev, F, W, nullptr, r->pipe_stream[k],
                                                     device_sm_count(), false));
                CUPBR_CHECK_CUDA(cudaEventRecord(r->pipe_traced[k], r->pipe_stream[k]));
                CUPBR_CHECK_CUDA(cudaStreamWaitEvent(r->stream, r->pipe_traced[k], 0));
                CUPBR_CHECK_CUDA(pt_launch_accumulate(F, W, r->hdr, r->stream));
                CUPBR_CHECK_CUDA(cudaEventRecord(r->pipe_folded[k], r->stream));
                ++r->frame;
                return CUPBR_OK;
            }
            CUPBR_CHECK_CUDA(r->pt.ensure(F.n_paths));
            if (r->instrumented) CUPBR_CHECK_CUDA(cudaMemsetAsync(r->pt.ws.stats, 0, sizeof(uint64_t) * STAT_TOTAL, r->stream));
            CUPBR_CHECK_CUDA(volume_render_frame(r->scene->g.dev, F, r->pt.ws, r->hdr, r->stream, device_sm_count(),
                                                 r->instrumented));
            if (r->instrumented) CUPBR_CHECK_CUDA(r->read_wavefront_rays());
            ++r->frame;
            return CUPBR_OK;
        }
        case CUPBR_GRADIENTDOMAIN:  // PBRenderer.cu:193-213
            return render_gdpt(r, cam, 1);
        case CUPBR_RAYTRACER: {  // PBRenderer.cu:154-159
            PTFrame F = make_frame(cam, r->w, r->h, 0, 0, false);
            CUPBR_CHECK_CUDA(launch_raytrace(r->scene->g.dev, F, r->hdr, r->pt.ws.err, r->stream));
            return CUPBR_OK;
        }
        case CUPBR_WHITTED: return fail(CUPBR_ERR_UNSUPPORTED, "WHITTED currently disabled.");  // PBRenderer.cu:161-170
        case CUPBR_METROPOLIS: return fail(CUPBR_ERR_UNSUPPORTED, "METROPOLIS not supported.");  // :187-191
        default: return fail(CUPBR_ERR_UNSUPPORTED, "unknown rendering method");
    }
}
cudaError_t cupbr_renderer_s::render_persistent(const cupbr_camera* c, uint32_t n) {
    cudaError_t e;
    const uint32_t pixels = w * h;
    if (!pk_scene || pk_w != w || pk_h != h) {
        pk_release();
        if ((e = dev_alloc(&pk_scene, sizeof(DeviceScene))) != cudaSuccess) return e;
        if ((e = dev_alloc(&pk_view, sizeof(BatchView))) != cudaSuccess) return e;
        if ((e = dev_alloc(&pk_counter, sizeof(uint32_t) * 2)) != cudaSuccess) return e;
        if ((e = cudaMemset(pk_counter, 0, sizeof(uint32_t) * 2)) != cudaSuccess) return e;
        std::vector<BatchItem> items;
        for (uint32_t s0 = 0; s0 < pixels; s0 += 32u) items.push_back(BatchItem{0u, s0});
        if ((e = dev_alloc(&pk_items, sizeof(BatchItem) * items.size())) != cudaSuccess) return e;
        if ((e = cudaMemcpy(pk_items, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return e;
        pk_items_n = (uint32_t)items.size();
        pk_w = w;
        pk_h = h;
    }
    if (pk_for != scene || pk_gen != scene->g.generation) {
        if ((e = cudaMemcpyAsync(pk_scene, &scene->g.dev, sizeof(DeviceScene), cudaMemcpyHostToDevice, stream)) !=
            cudaSuccess)
            return e;
        pk_for = scene;
        pk_gen = scene->g.generation;
    }
    BatchView v;
    v.cam_pos = mk(c->position.x, c->position.y, c->position.z);
    v.cam_x = mk(c->x_axis.x, c->x_axis.y, c->x_axis.z);
    v.cam_y = mk(c->y_axis.x, c->y_axis.y, c->y_axis.z);
    v.cam_z = mk(c->z_axis.x, c->z_axis.y, c->z_axis.z);
    v.width = w;
    v.height = h;
    v.frame0 = frame;
    v.spp = n;
    v.img = hdr;
    v.scene = 0;
    if ((e = cudaMemcpyAsync(pk_view, &v, sizeof v, cudaMemcpyHostToDevice, stream)) != cudaSuccess) return e;
    // the host copy of v is pageable: the copy is done when the call returns
    return batch_launch_persistent(pk_scene, pk_view, pk_items, pk_items_n, pk_counter, max_depth, 128,
                                   (uint32_t)batch_persistent_occupancy(128, true), true, device_sm_count(),
                                   pk_counter + 1, stream);
}

int cupbr_renderer_set_persistent(cupbr_renderer_t r, int32_t enable) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    r->persistent = enable != 0;
    return CUPBR_OK;
}
int cupbr_renderer_render_frames(cupbr_renderer_t r, const cupbr_camera* cam, uint32_t nframes) {
    NvtxRange nvtx_("cupbr_renderer_render_frames");
    if (!r || !cam) return fail(CUPBR_ERR_ARG, "null argument");
    if (r->method == CUPBR_GRADIENTDOMAIN && r->size_set && r->scene) {
        if (nframes == 0) return CUPBR_OK;
        return render_gdpt(r, cam, nframes);
    }
    if (r->method == CUPBR_VOLUME && !r->instrumented && r->size_set && r->scene && r->max_depth <= PT_MAX_DEPTH) {
        // VOLUME frames as multi-frame wavefronts (frame index and running
        // mean per frame as render() gives them)
        if (cam->moved) r->frame = 0;
        const uint32_t pixels = r->w * r->h;
        const uint32_t per = std::max(1u, std::min(nframes, r->batch_paths / std::max(1u, pixels)));
        CUPBR_CHECK_CUDA(r->pt.ensure(per * pixels));
        for (uint32_t done = 0; done < nframes;) {
            const uint32_t k = std::min(per, nframes - done);
            PTFrame F = make_frame(cam, r->w, r->h, r->frame, r->max_depth, r->rr, r->estimator);
            F.frames = k;
            F.n_paths = k * pixels;
            CUPBR_CHECK_CUDA(volume_render_frame(r->scene->g.dev, F, r->pt.ws, r->hdr, r->stream, device_sm_count(),
                                                 false));
            r->frame += k;
            done += k;
        }
        return CUPBR_OK;
    }
    if (r->method != CUPBR_PATHTRACER || r->instrumented) {
        cupbr_camera still = *cam;  // only the first frame may restart accumulation
        still.moved = 0;
        for (uint32_t i = 0; i < nframes; ++i) {
            int s = cupbr_renderer_render(r, i == 0 ? cam : &still);
            if (s != CUPBR_OK) return s;
        }
        return CUPBR_OK;
    }
    if (!r->size_set) return fail(CUPBR_ERR_STATE, "No output size set. Use setOutputSize()");
    if (!r->scene) return fail(CUPBR_ERR_STATE, "No scene registered. Use registerScene()");
    if (r->max_depth > PT_MAX_DEPTH) return fail(CUPBR_ERR_ARG, "max trace depth above 64");
    if (cam->moved) r->frame = 0;
    if (r->persistent && !r->rr && r->estimator == CUPBR_ESTIMATOR_REFERENCE && !r->profiling && nframes) {
        CUPBR_CHECK_CUDA(r->render_persistent(cam, nframes));
        r->frame += nframes;
        return CUPBR_OK;
    }
    const uint32_t pixels = r->w * r->h;
    uint32_t per = std::max(1u, std::min(nframes, r->batch_paths / pixels));
    if (r->pipelined && !r->profiling) {
        // wavefronts alternate between the two internal streams and
        // workspaces, so one wavefront's last, sparse depths overlap the
        // next one's first; each is folded into the image on the caller's
        // stream in frame order (the same image as one stream)
        CUPBR_CHECK_CUDA(r->pipe_init());
        for (int k = 0; k < 2; ++k) CUPBR_CHECK_CUDA(r->pipe_pt[k].ensure(per * pixels));
        // the call's wavefronts start after the work already queued on the
        // caller's stream (scene edits, image resets, a timing event)
        CUPBR_CHECK_CUDA(cudaEventRecord(r->pipe_start, r->stream));
        for (int k = 0; k < 2; ++k) CUPBR_CHECK_CUDA(cudaStreamWaitEvent(r->pipe_stream[k], r->pipe_start, 0));
        for (uint32_t done = 0; done < nframes;) {
            const uint32_t n = std::min(per, nframes - done);
            PTFrame F = make_frame(cam, r->w, r->h, r->frame, r->max_depth, r->rr, r->estimator);
            F.frames = n;
            F.n_paths = n * pixels;
            const uint32_t k = r->pipe_next % 2u;
            r->pipe_next = k ^ 1u;
            const Workspace& W = r->pipe_pt[k].ws;
            CUPBR_CHECK_CUDA(cudaStreamWaitEvent(r->pipe_stream[k], r->pipe_folded[k], 0));
            CUPBR_CHECK_CUDA(pt_render_frame(r->scene->g.dev, F, W, nullptr, r->pipe_stream[k], device_sm_count(),
                                             false, nullptr, r->tail()));
            CUPBR_CHECK_CUDA(cudaEventRecord(r->pipe_traced[k], r->pipe_stream[k]));
            CUPBR_CHECK_CUDA(cudaStreamWaitEvent(r->stream, r->pipe_traced[k], 0));
            CUPBR_CHECK_CUDA(pt_launch_accumulate(F, W, r->hdr, r->stream));
            CUPBR_CHECK_CUDA(cudaEventRecord(r->pipe_folded[k], r->stream));
            r->frame += n;
            done += n;
        }
        return CUPBR_OK;
    }
    if (per > 1) CUPBR_CHECK_CUDA(r->pt.ensure(per * pixels));
    for (uint32_t done = 0; done < nframes;) {
        const uint32_t k = std::min(per, nframes - done);
        PTFrame F = make_frame(cam, r->w, r->h, r->frame, r->max_depth, r->rr, r->estimator);
        F.frames = k;
        F.n_paths = k * pixels;
        std::vector<cudaEvent_t> ev;
        if (r->profiling) CUPBR_CHECK_CUDA(r->events.take(pt_event_count(r->max_depth), ev));
        CUPBR_CHECK_CUDA(pt_render_frame(r->scene->g.dev, F, r->pt.ws, r->hdr, r->stream, device_sm_count(), false,
                                         r->profiling ? ev.data() : nullptr, r->tail()));
        if (r->profiling) r->events.frames.push_back({std::move(ev), 3u});
        r->frame += k;
        done += k;
    }
    return CUPBR_OK;
}
int cupbr_renderer_set_batch_paths(cupbr_renderer_t r, uint32_t paths) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    r->batch_paths = std::max(1u, paths);
    return CUPBR_OK;
}
int cupbr_renderer_reset(cupbr_renderer_t r) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    r->frame = 0;
    return CUPBR_OK;
}
int cupbr_renderer_set_tail_paths(cupbr_renderer_t r, uint32_t paths) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    r->tail_paths = paths;
    r->tail_set = true;
    return CUPBR_OK;
}
int cupbr_renderer_set_russian_roulette(cupbr_renderer_t r, int32_t enable) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    r->rr = enable != 0;
    return CUPBR_OK;
}
int cupbr_renderer_set_max_trace_depth(cupbr_renderer_t r, uint32_t d) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    if (d > PT_MAX_DEPTH) return fail(CUPBR_ERR_ARG, "max trace depth above 64");
    r->max_depth = d;
    return CUPBR_OK;
}
int cupbr_renderer_get_max_trace_depth(cupbr_renderer_t r, uint32_t* d) {
    if (!r || !d) return fail(CUPBR_ERR_ARG, "null argument");
    *d = r->max_depth;
    return CUPBR_OK;
}
int cupbr_renderer_get_output(cupbr_renderer_t r, float** dev, uint32_t* w, uint32_t* h) {
    if (!r || !dev) return fail(CUPBR_ERR_ARG, "null argument");
    *dev = r->hdr;
    if (w) *w = r->w;
    if (h) *h = r->h;
    return CUPBR_OK;
}
int cupbr_renderer_get_gradient_x(cupbr_renderer_t r, float** dev) {
    if (!r || !dev) return fail(CUPBR_ERR_ARG, "null argument");
    *dev = r->aux.size() > 0 ? r->aux[0] : nullptr;
    return CUPBR_OK;
}
int cupbr_renderer_get_gradient_y(cupbr_renderer_t r, float** dev) {
    if (!r || !dev) return fail(CUPBR_ERR_ARG, "null argument");
    *dev = r->aux.size() > 1 ? r->aux[1] : nullptr;
    return CUPBR_OK;
}
int cupbr_gdpt_reconstruct(uint32_t w, uint32_t h, const float* base, const float* gxf, const float* gxb,
                           const float* gyf, const float* gyb, float* gx, float* gy, float* temp, float* out,
                           void* stream) {
    if (!base || !gxf || !gxb || !gyf || !gyb || !gx || !gy || !temp || !out) return fail(CUPBR_ERR_ARG, "null buffer");
    if ((uint64_t)w * h >= (1ull << 31)) return fail(CUPBR_ERR_ARG, "image too large");
    CUPBR_CHECK_CUDA(launch_gdpt_reconstruct(w, h, base, gxf, gxb, gyf, gyb, gx, gy, temp, out, (cudaStream_t)stream));
    return CUPBR_OK;
}
int cupbr_renderer_get_frame_index(cupbr_renderer_t r, uint32_t* f) {
    if (!r || !f) return fail(CUPBR_ERR_ARG, "null argument");
    *f = r->frame;
    return CUPBR_OK;
}
int cupbr_renderer_set_frame_index(cupbr_renderer_t r, uint32_t f) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    r->frame = f;
    return CUPBR_OK;
}
int cupbr_renderer_set_stream(cupbr_renderer_t r, void* stream) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    r->stream = (cudaStream_t)stream;
    return CUPBR_OK;
}
int cupbr_renderer_get_error_count(cupbr_renderer_t r, uint32_t* count) {
    if (!r || !count) return fail(CUPBR_ERR_ARG, "null argument");
    *count = 0;
    constexpr int NS = cupbr_renderer_s::PIPE_SLOTS;
    const uint32_t* bufs[1 + NS] = {r->pt.ws.err};
    for (int k = 0; k < NS; ++k) bufs[1 + k] = r->pipe_pt[k].ws.err;
    for (int k = 0; k < 1 + NS; ++k) {
        if (k > 0 && r->pipe_stream[k - 1]) CUPBR_CHECK_CUDA(cudaStreamSynchronize(r->pipe_stream[k - 1]));
        if (!bufs[k]) continue;
        uint32_t e[ERR_TOTAL];
        CUPBR_CHECK_CUDA(cudaMemcpyAsync(e, bufs[k], sizeof e, cudaMemcpyDeviceToHost, r->stream));
        CUPBR_CHECK_CUDA(cudaStreamSynchronize(r->stream));
        for (uint32_t j = 0; j < ERR_TOTAL; ++j) *count += e[j];
    }
    if (r->pk_counter) {
        uint32_t e = 0;
        CUPBR_CHECK_CUDA(cudaMemcpyAsync(&e, r->pk_counter + 1, sizeof e, cudaMemcpyDeviceToHost, r->stream));
        CUPBR_CHECK_CUDA(cudaStreamSynchronize(r->stream));
        *count += e;
    }
    return CUPBR_OK;
}
int cupbr_renderer_set_pipelined(cupbr_renderer_t r, int32_t enable) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    r->pipelined = enable != 0;
    return CUPBR_OK;
}
int cupbr_renderer_set_instrumented(cupbr_renderer_t r, int32_t enable) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    r->instrumented = enable != 0;
    return CUPBR_OK;
}
int cupbr_renderer_set_profiling(cupbr_renderer_t r, int32_t enable) {
    if (!r) return fail(CUPBR_ERR_ARG, "null renderer");
    r->profiling = enable != 0;
    if (r->profiling) CUPBR_CHECK_CUDA(r->events.reserve(4096));
    return CUPBR_OK;
}
int cupbr_renderer_get_stage_times(cupbr_renderer_t r, float* ms5, uint32_t* frames, uint32_t* launches) {
    if (!r || !ms5) return fail(CUPBR_ERR_ARG, "null argument");
    CUPBR_CHECK_CUDA(r->events.read(ms5, 3, frames, launches));
    return CUPBR_OK;
}
int cupbr_renderer_get_stats(cupbr_renderer_t r, uint64_t* st) {
    if (!r || !st) return fail(CUPBR_ERR_ARG, "null argument");
    if (!r->pt.ws.stats) return fail(CUPBR_ERR_STATE, "no output size set");
    CUPBR_CHECK_CUDA(cudaMemcpyAsync(st, r->pt.ws.stats, sizeof(uint64_t) * STAT_TOTAL, cudaMemcpyDeviceToHost, r->stream));
    CUPBR_CHECK_CUDA(cudaStreamSynchronize(r->stream));
    st[4] = r->last_rays[0];
    st[5] = r->last_rays[1];
    return CUPBR_OK;
}

int cupbr_pathtracing(cupbr_scene_t s, const cupbr_camera* cam, uint32_t frame, uint32_t depth, int32_t rr,
                      float* img, uint32_t w, uint32_t h, void* stream) {
    if (!s || !cam || !img) return fail(CUPBR_ERR_ARG, "null argument");
    if (!s->g.committed) return fail(CUPBR_ERR_STATE, "scene not committed");
    if (w == 0 || h == 0 || (uint64_t)w * h >= (1ull << 30)) return fail(CUPBR_ERR_ARG, "bad image size");
    if (depth > PT_MAX_DEPTH) return fail(CUPBR_ERR_ARG, "max trace depth above 64");
    CUPBR_CHECK_CUDA(s->pt.ensure(w * h));
    PTFrame F = make_frame(cam, w, h, frame, depth, rr != 0);
    CUPBR_CHECK_CUDA(pt_render_frame(s->g.dev, F, s->pt.ws, img, (cudaStream_t)stream, device_sm_count(), false, nullptr));
    return CUPBR_OK;
}

// ----------------------------------------------------------- tone map ---
int cupbr_tonemapper_create(int32_t type, cupbr_tonemapper_t* out) {
    if (!out) return fail(CUPBR_ERR_ARG, "null output");
    if (type != CUPBR_REINHARD && type != CUPBR_GAMMA) return fail(CUPBR_ERR_ARG, "unknown tone mapping type");
    cupbr_tonemapper_s* t = new cupbr_tonemapper_s();
    t->type = type;
    *out = t;
    return CUPBR_OK;
}
int cupbr_tonemapper_destroy(cupbr_tonemapper_t t) {
    delete t;
    return CUPBR_OK;
}
int cupbr_tonemapper_register_image(cupbr_tonemapper_t t, const float* hdr, uint32_t w, uint32_t h) {
    if (!t || !hdr || w == 0 || h == 0) return fail(CUPBR_ERR_ARG, "bad argument");
    if (t->rgba) cudaFree(t->rgba);
    t->rgba = nullptr;
    CUPBR_CHECK_CUDA(dev_alloc(&t->rgba, 4 * (size_t)w * h));
    t->hdr = hdr;
    t->w = w;
    t->h = h;
    return CUPBR_OK;
}
int cupbr_tonemapper_tonemap(cupbr_tonemapper_t t) {
    if (!t) return fail(CUPBR_ERR_ARG, "null tone mapper");
    if (!t->hdr) return fail(CUPBR_ERR_STATE, "No HDR image has been registered. Call registerImage() first!");
    CUPBR_CHECK_CUDA(launch_tonemap(t->hdr, t->w * t->h, t->type, t->exposure, t->rgba, t->stream));
    return CUPBR_OK;
}
int cupbr_tonemapper_get_render_buffer(cupbr_tonemapper_t t, uint8_t** dev, uint32_t* w, uint32_t* h) {
    if (!t || !dev) return fail(CUPBR_ERR_ARG, "null argument");
    *dev = t->rgba;
    if (w) *w = t->w;
    if (h) *h = t->h;
    return CUPBR_OK;
}
int cupbr_tonemapper_get_type(cupbr_tonemapper_t t, int32_t* type) {
    if (!t || !type) return fail(CUPBR_ERR_ARG, "null argument");
    *type = t->type;
    return CUPBR_OK;
}
int cupbr_tonemapper_set_type(cupbr_tonemapper_t t, int32_t type) {
    if (!t) return fail(CUPBR_ERR_ARG, "null tone mapper");
    if (type != CUPBR_REINHARD && type != CUPBR_GAMMA) return fail(CUPBR_ERR_ARG, "unknown tone mapping type");
    t->type = type;
    return CUPBR_OK;
}
int cupbr_tonemapper_set_exposure(cupbr_tonemapper_t t, float e) {
    if (!t) return fail(CUPBR_ERR_ARG, "null tone mapper");
    t->exposure = e;
    return CUPBR_OK;
}
int cupbr_tonemapper_set_stream(cupbr_tonemapper_t t, void* stream) {
    if (!t) return fail(CUPBR_ERR_ARG, "null tone mapper");
    t->stream = (cudaStream_t)stream;
    return CUPBR_OK;
}
int cupbr_tonemapper_save_to_file(cupbr_tonemapper_t t, const char* path) {
    if (!t || !path) return fail(CUPBR_ERR_ARG, "null argument");
    if (!t->rgba) return fail(CUPBR_ERR_STATE, "no render buffer");
    std::vector<uint8_t> host(4 * (size_t)t->w * t->h);
    CUPBR_CHECK_CUDA(cudaMemcpyAsync(host.data(), t->rgba, host.size(), cudaMemcpyDeviceToHost, t->stream));
    CUPBR_CHECK_CUDA(cudaStreamSynchronize(t->stream));
    std::string err;
    if (!write_bmp_rgba(path, host.data(), t->w, t->h, false, err)) return fail(CUPBR_ERR_IO, err);
    return CUPBR_OK;
}
int cupbr_tonemap(const float* hdr, uint32_t w, uint32_t h, int32_t type, float exposure, uint8_t* rgba, void* stream) {
    if (!hdr || !rgba) return fail(CUPBR_ERR_ARG, "null argument");
    if (type != CUPBR_REINHARD && type != CUPBR_GAMMA) return fail(CUPBR_ERR_ARG, "unknown tone mapping type");
    CUPBR_CHECK_CUDA(launch_tonemap(hdr, w * h, type, exposure, rgba, (cudaStream_t)stream));
    return CUPBR_OK;
}

int cupbr_tonemap_verify_levels(uint64_t mismatches[3], uint32_t flagged[3], void* stream) {
    if (!mismatches || !flagged) return fail(CUPBR_ERR_ARG, "null argument");
    unsigned long long m[3] = {0, 0, 0};
    CUPBR_CHECK_CUDA(verify_tone_levels(m, flagged, (cudaStream_t)stream));
    for (int t = 0; t < 3; ++t) mismatches[t] = m[t];
    return CUPBR_OK;
}

// ------------------------------------------------------- post process ---
int cupbr_postprocessor_create(cupbr_postprocessor_t* out) {
    if (!out) return fail(CUPBR_ERR_ARG, "null output");
    *out = new cupbr_postprocessor_s();
    return CUPBR_OK;
}
int cupbr_postprocessor_destroy(cupbr_postprocessor_t p) {
    delete p;
    return CUPBR_OK;
}
int cupbr_postprocessor_register_image(cupbr_postprocessor_t p, const float* hdr, uint32_t w, uint32_t h) {
    if (!p || !hdr) return fail(CUPBR_ERR_ARG, "null argument");
    if (w < 2 || h < 2) return fail(CUPBR_ERR_ARG, "bloom needs an image of at least 2x2 pixels");
    if (p->out) cudaFree(p->out);
    if (p->half) cudaFree(p->half);
    p->out = p->half = nullptr;
    CUPBR_CHECK_CUDA(dev_alloc(&p->out, sizeof(float) * 3 * (size_t)w * h));
    CUPBR_CHECK_CUDA(dev_alloc(&p->half, sizeof(float) * 3 * (size_t)(w / 2) * (h / 2)));
    p->hdr = hdr;
    p->w = w;
    p->h = h;
    return CUPBR_OK;
}
int cupbr_postprocessor_get_buffer(cupbr_postprocessor_t p, float** dev) {
    if (!p || !dev) return fail(CUPBR_ERR_ARG, "null argument");
    *dev = p->out;
    return CUPBR_OK;
}
int cupbr_postprocessor_bloom(cupbr_postprocessor_t p, const float th[4]) {
    NvtxRange nvtx_("cupbr_postprocessor_bloom");
    if (!p || !th) return fail(CUPBR_ERR_ARG, "null argument");
    if (!p->hdr) return fail(CUPBR_ERR_STATE, "no image registered");
    CUPBR_CHECK_CUDA(launch_bloom(p->hdr, p->w, p->h, th, p->half, p->out, nullptr, 0, 0.0f, p->stream));
    return CUPBR_OK;
}
int cupbr_postprocessor_bloom_tonemap(cupbr_postprocessor_t p, const float th[4], int32_t type, float exposure,
                                      uint8_t* rgba) {
    NvtxRange nvtx_("cupbr_postprocessor_bloom_tonemap");
    if (!p || !th || !rgba) return fail(CUPBR_ERR_ARG, "null argument");
    if (!p->hdr) return fail(CUPBR_ERR_STATE, "no image registered");
    if (type != CUPBR_REINHARD && type != CUPBR_GAMMA) return fail(CUPBR_ERR_ARG, "unknown tone mapping type");
    CUPBR_CHECK_CUDA(launch_bloom(p->hdr, p->w, p->h, th, p->half, nullptr, rgba, type, exposure, p->stream));
    return CUPBR_OK;
}
// Bloom for callers that cannot allocate device memory: the level-1 scratch
// is a fixed array inside the library (post.cu), so this call performs no
// cudaMalloc / cudaFree.  Its first call on a device looks up that array's
// device address.
int cupbr_bloom_noalloc(const float* hdr, uint32_t w, uint32_t h, const float th[4], float* out, void* stream) {
    if (!hdr || !th || !out) return fail(CUPBR_ERR_ARG, "null argument");
    if (w < 2 || h < 2) return fail(CUPBR_ERR_ARG, "bloom needs an image of at least 2x2 pixels");
    if ((uint64_t)(w / 2) * (h / 2) > BLOOM_NOALLOC_MAX_HALF_PIXELS)
        return fail(CUPBR_ERR_ARG, "image too large for the fixed bloom scratch: (width/2)*(height/2) must be at most " +
                                       std::to_string(BLOOM_NOALLOC_MAX_HALF_PIXELS) + " (e.g. 2048x2048)");
    CUPBR_CHECK_CUDA(bloom_static_scratch(hdr, w, h, th, out, (cudaStream_t)stream));
    return CUPBR_OK;
}
int cupbr_postprocessor_set_stream(cupbr_postprocessor_t p, void* stream) {
    if (!p) return fail(CUPBR_ERR_ARG, "null post processor");
    p->stream = (cudaStream_t)stream;
    return CUPBR_OK;
}

// ------------------------------------------------- heterogeneous medium ---
struct cupbr_medium_s {
    cupbr_medium_desc desc{};
    uint32_t* err = nullptr;  // one device counter, zeroed at creation
    PTBuffers pt;             // wavefront queues (shared with the path tracer's layout)
    float4* aux = nullptr;    // per shadow-queue slot: ratio-tracking RNG state, light, Lambert object
    double* lsum = nullptr;   // 3 per path (gradient replays)
    float4* verts = nullptr;  // 3 per path: a depth's medium and surface vertices
    uint32_t aux_capacity = 0;
    uint32_t batch_paths = 1u << 22;  // paths per wavefront
    bool profiling = false, instrumented = false;
    StageEvents events;
    unsigned long long* stats = nullptr;  // 4 device counters (see MediumWorkspace)
    ~cupbr_medium_s() {
        if (err) cudaFree(err);
        if (aux) cudaFree(aux);
        if (lsum) cudaFree(lsum);
        if (verts) cudaFree(verts);
        if (stats) cudaFree(stats);
    }
    cudaError_t ensure(uint32_t pixels, uint32_t spp, MediumWorkspace& W) {
        const uint64_t want = std::max<uint64_t>(pixels, std::min<uint64_t>((uint64_t)pixels * spp, batch_paths));
        const uint32_t n = (uint32_t)std::min<uint64_t>(want, 0xFFFFFFFFull);
        cudaError_t e = pt.ensure(n);
        if (e != cudaSuccess) return e;
        if (aux_capacity < pt.capacity) {
            if (aux) cudaFree(aux);
            if (lsum) cudaFree(lsum);
            if (verts) cudaFree(verts);
            aux = nullptr;
            lsum = nullptr;
            verts = nullptr;
            aux_capacity = 0;
            if ((e = dev_alloc(&aux, sizeof(float4) * (size_t)pt.capacity)) != cudaSuccess) return e;
            if ((e = dev_alloc(&lsum, sizeof(double) * 3 * (size_t)pt.capacity)) != cudaSuccess) return e;
            if ((e = dev_alloc(&verts, sizeof(float4) * 3 * (size_t)pt.capacity)) != cudaSuccess) return e;
            aux_capacity = pt.capacity;
        }
        W.pt = pt.ws;
        W.shadow_aux = aux;
        W.lsum = lsum;
        W.verts = verts;
        W.capacity = pt.capacity;
        W.stats = nullptr;
        if (instrumented) {
            if (!stats) {
                if ((e = dev_alloc(&stats, MEDIUM_STATS * sizeof(unsigned long long))) != cudaSuccess) return e;
                if ((e = cudaMemset(stats, 0, MEDIUM_STATS * sizeof(unsigned long long))) != cudaSuccess) return e;
            }
            W.stats = stats;
        }
        return cudaSuccess;
    }
};

int cupbr_medium_create(const cupbr_medium_desc* d, cupbr_medium_t* out) {
    if (!d || !out) return fail(CUPBR_ERR_ARG, "null argument");
    if (d->nx == 0 || d->ny == 0 || d->nz == 0) return fail(CUPBR_ERR_ARG, "empty density grid");
    if ((uint64_t)d->nx * d->ny * d->nz > 0xFFFFFFFFull) return fail(CUPBR_ERR_ARG, "density grid too large");
    if (!(d->lo.x < d->hi.x && d->lo.y < d->hi.y && d->lo.z < d->hi.z)) return fail(CUPBR_ERR_ARG, "empty grid box");
    if (!(d->majorant > 0.0f) || !std::isfinite(d->majorant)) return fail(CUPBR_ERR_ARG, "majorant must be positive");
    if (!(d->albedo >= 0.0f && d->albedo <= 1.0f)) return fail(CUPBR_ERR_ARG, "albedo must lie in [0, 1]");
    if (!(std::fabs(d->g) < 1.0f)) return fail(CUPBR_ERR_ARG, "|g| must be below 1");
    if (!(d->q >= 0.0f && d->q < 1.0f)) return fail(CUPBR_ERR_ARG, "q must lie in [0, 1)");
    std::unique_ptr<cupbr_medium_s> m(new cupbr_medium_s());
    m->desc = *d;
    CUPBR_CHECK_CUDA(dev_alloc(&m->err, sizeof(uint32_t)));
    CUPBR_CHECK_CUDA(cudaMemset(m->err, 0, sizeof(uint32_t)));
    *out = m.release();
    return CUPBR_OK;
}
int cupbr_medium_destroy(cupbr_medium_t m) {
    delete m;
    return CUPBR_OK;
}
int cupbr_medium_param_count(cupbr_scene_t s, uint32_t* out) {
    if (!s || !out) return fail(CUPBR_ERR_ARG, "null argument");
    *out = medium_param_count((uint32_t)s->g.host.objects.size(), (uint32_t)s->g.host.lights.size());
    return CUPBR_OK;
}

static int medium_setup(cupbr_medium_t m, cupbr_scene_t s, const float* density, const cupbr_camera* cam, uint32_t w,
                        uint32_t h, uint32_t spp, uint32_t frame0, uint32_t depth, MediumGrid& G, MediumParams& P) {
    if (!m || !s || !density || !cam) return fail(CUPBR_ERR_ARG, "null argument");
    if (!s->g.committed) return fail(CUPBR_ERR_STATE, "scene not committed");
    if ((uint64_t)w * h > 0xFFFFFFFFull / 3) return fail(CUPBR_ERR_ARG, "image too large");
    if (spp == 0) return fail(CUPBR_ERR_ARG, "spp must be at least 1");
    if (depth == 0 || depth > PT_MAX_DEPTH)
        return fail(CUPBR_ERR_ARG, "max_depth must lie in [1, " + std::to_string(PT_MAX_DEPTH) + "]");
    const cupbr_medium_desc& d = m->desc;
    G.density = density;
    G.nx = d.nx;
    G.ny = d.ny;
    G.nz = d.nz;
    G.lo = mk(d.lo.x, d.lo.y, d.lo.z);
    G.hi = mk(d.hi.x, d.hi.y, d.hi.z);
    G.inv_cell = mk((float)d.nx / (d.hi.x - d.lo.x), (float)d.ny / (d.hi.y - d.lo.y), (float)d.nz / (d.hi.z - d.lo.z));
    G.majorant = d.majorant;
    G.inv_majorant = 1.0f / d.majorant;
    P.width = w;
    P.height = h;
    P.spp = spp;
    P.frame0 = frame0;
    P.max_depth = depth;
    P.albedo = d.albedo;
    P.g = d.g;
    P.q = d.q;
    P.inv_q = d.q > 0.0f ? 1.0f / d.q : 0.0f;
    P.inv_one_minus_q = 1.0f / (1.0f - d.q);
    P.cam_pos = mk(cam->position.x, cam->position.y, cam->position.z);
    P.cam_x = mk(cam->x_axis.x, cam->x_axis.y, cam->x_axis.z);
    P.cam_y = mk(cam->y_axis.x, cam->y_axis.y, cam->y_axis.z);
    P.cam_z = mk(cam->z_axis.x, cam->z_axis.y, cam->z_axis.z);
    return CUPBR_OK;
}

int cupbr_medium_forward(cupbr_medium_t m, cupbr_scene_t s, const float* density, const cupbr_camera* cam, uint32_t w,
                         uint32_t h, uint32_t spp, uint32_t frame0, uint32_t depth, float* image, void* stream) {
    NvtxRange nvtx_("cupbr_medium_forward");
    MediumGrid G;
    MediumParams P;
    if (int rc = medium_setup(m, s, density, cam, w, h, spp, frame0, depth, G, P)) return rc;
    if (!image) return fail(CUPBR_ERR_ARG, "null image");
    MediumWorkspace W;
    CUPBR_CHECK_CUDA(m->ensure(w * h, spp, W));
    std::vector<cudaEvent_t> ev;
    const uint32_t nb = medium_batches(P, W);
    if (m->profiling) CUPBR_CHECK_CUDA(m->events.take(nb * medium_event_count(depth), ev));
    CUPBR_CHECK_CUDA(medium_render(s->g.dev, G, P, W, image, m->err, device_sm_count(), (cudaStream_t)stream,
                                   m->profiling ? ev.data() : nullptr));
    if (m->profiling) {
        const size_t per = medium_event_count(depth);
        for (uint32_t b = 0; b < nb; ++b)
            m->events.frames.push_back({std::vector<cudaEvent_t>(ev.begin() + b * per, ev.begin() + (b + 1) * per), 4u});
    }
    return CUPBR_OK;
}
int cupbr_medium_backward(cupbr_medium_t m, cupbr_scene_t s, const float* density, const cupbr_camera* cam, uint32_t w,
                          uint32_t h, uint32_t spp, uint32_t frame0, uint32_t depth, const float* grad_image,
                          float* grad_density, float* grad_params, void* stream) {
    NvtxRange nvtx_("cupbr_medium_backward");
    MediumGrid G;
    MediumParams P;
    if (int rc = medium_setup(m, s, density, cam, w, h, spp, frame0, depth, G, P)) return rc;
    if (!grad_image || !grad_density || !grad_params) return fail(CUPBR_ERR_ARG, "null gradient buffer");
    if (!(m->desc.q > 0.0f)) return fail(CUPBR_ERR_UNSUPPORTED, "gradients need weighted tracking (0 < q < 1)");
    MediumWorkspace W;
    CUPBR_CHECK_CUDA(m->ensure(w * h, spp, W));
    CUPBR_CHECK_CUDA(medium_gradient(s->g.dev, G, P, W, grad_image, grad_density, grad_params, m->err,
                                     device_sm_count(), (cudaStream_t)stream));
    return CUPBR_OK;
}
int cupbr_medium_set_batch_paths(cupbr_medium_t m, uint32_t paths) {
    if (!m || paths == 0) return fail(CUPBR_ERR_ARG, "batch must hold at least one path");
    m->batch_paths = paths;
    return CUPBR_OK;
}
int cupbr_medium_set_profiling(cupbr_medium_t m, int32_t enable) {
    if (!m) return fail(CUPBR_ERR_ARG, "null medium");
    m->profiling = enable != 0;
    if (m->profiling) CUPBR_CHECK_CUDA(m->events.reserve(4096));
    return CUPBR_OK;
}
int cupbr_medium_get_stage_times(cupbr_medium_t m, float* ms6, uint32_t* wavefronts, uint32_t* shade_launches) {
    if (!m || !ms6) return fail(CUPBR_ERR_ARG, "null argument");
    CUPBR_CHECK_CUDA(m->events.read(ms6, 4, wavefronts, shade_launches));
    return CUPBR_OK;
}
int cupbr_medium_set_instrumented(cupbr_medium_t m, int32_t enable) {
    if (!m) return fail(CUPBR_ERR_ARG, "null medium");
    m->instrumented = enable != 0;
    return CUPBR_OK;
}
int cupbr_medium_get_stats(cupbr_medium_t m, uint64_t* stats5) {
    if (!m || !stats5) return fail(CUPBR_ERR_ARG, "null argument");
    for (uint32_t k = 0; k < MEDIUM_STATS; ++k) stats5[k] = 0;
    if (!m->stats) return CUPBR_OK;
    unsigned long long v[MEDIUM_STATS];
    CUPBR_CHECK_CUDA(cudaDeviceSynchronize());
    CUPBR_CHECK_CUDA(cudaMemcpy(v, m->stats, sizeof v, cudaMemcpyDeviceToHost));
    CUPBR_CHECK_CUDA(cudaMemset(m->stats, 0, sizeof v));
    for (uint32_t k = 0; k < MEDIUM_STATS; ++k) stats5[k] = v[k];
    return CUPBR_OK;
}
int cupbr_medium_get_error_count(cupbr_medium_t m, uint32_t* out) {
    if (!m || !out) return fail(CUPBR_ERR_ARG, "null argument");
    CUPBR_CHECK_CUDA(cudaDeviceSynchronize());
    CUPBR_CHECK_CUDA(cudaMemcpy(out, m->err, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (m->pt.ws.err) {
        uint32_t e[ERR_TOTAL];
        CUPBR_CHECK_CUDA(cudaMemcpy(e, m->pt.ws.err, sizeof e, cudaMemcpyDeviceToHost));
        for (uint32_t k = 0; k < ERR_TOTAL; ++k) *out += e[k];
    }
    return CUPBR_OK;
}

// ------------------------------------------------------ batched views ---
struct cupbr_batch_s {
    std::vector<cupbr_scene_s*> scenes;  // distinct scenes, first-use order
    std::vector<uint32_t> view_scene;    // per view: index into scenes
    std::vector<BatchView> views;        // host copy of the device table
    uint32_t max_depth = 5;
    uint32_t batch_paths = 1u << 22;
    float trace_share = 1.0f;            // fraction of the traversal kernels' full occupancy
    PTBuffers pt;
    std::vector<BatchWave> waves;
    std::vector<BatchSegment> segs;
    BatchView* dviews = nullptr;
    BatchSegment* dsegs = nullptr;
    cudaStream_t cap = nullptr;          // capture stream
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool dirty = true;                   // device view table out of date
    uint32_t launches_per_replay = 0;
    // CUPBR_BATCH_PERSISTENT: one launch of the persistent kernel over all
    // views (work items heaviest first); CUPBR_BATCH_WAVEFRONT: per scene a
    // sequence of wavefronts of at most batch_paths paths;
    // CUPBR_BATCH_COOPERATIVE: the same wavefronts in one cooperative launch
    int32_t mode = CUPBR_BATCH_PERSISTENT;
    uint32_t pers_threads = 128;         // threads per block of the persistent kernel
    uint32_t pers_blocks = 0;            // blocks per SM (0: as many as fit)
    bool pers_packets = true;            // camera rays of a frame as one warp packet
    std::vector<uint64_t> scene_gen;     // the scenes' commit generations the tables and graph were built for
    DeviceScene* dscenes = nullptr;      // the scenes' device records
    BatchItem* ditems = nullptr;
    uint32_t n_items = 0;
    uint32_t* dcounter = nullptr;        // [0] item counter, [1] traversal stack overflows
    BatchWave* dwaves = nullptr;         // cooperative mode: the wavefront table
    BatchBarrier* dbar = nullptr;        // cooperative mode: grid barrier (abort = a barrier timed out)
    uint64_t barrier_probe_ns = 0;       // cooperative mode test hook (cupbr_batch_set_barrier_probe)
    // albedo-texture adjoint: per scene its gradient (tex_w * tex_h RGB,
    // null for untextured scenes), and the device pointer tables of a call
    std::vector<float*> tex_grad;
    const float** dgrad_img = nullptr;
    float** dgrad_tex = nullptr;
    ~cupbr_batch_s() {
        release_graph();
        free_tables();
        for (float* g : tex_grad) if (g) cudaFree(g);
        if (dgrad_img) cudaFree(dgrad_img);
        if (dgrad_tex) cudaFree(dgrad_tex);
        if (cap) cudaStreamDestroy(cap);
    }
    void release_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    void free_tables() {
        if (dviews) cudaFree(dviews);
        if (dsegs) cudaFree(dsegs);
        if (dscenes) cudaFree(dscenes);
        if (ditems) cudaFree(ditems);
        if (dcounter) cudaFree(dcounter);
        if (dwaves) cudaFree(dwaves);
        if (dbar) cudaFree(dbar);
        dwaves = nullptr;
        dbar = nullptr;
        dviews = nullptr;
        dsegs = nullptr;
        dscenes = nullptr;
        ditems = nullptr;
        dcounter = nullptr;
    }
    uint32_t blocks_per_sm() const {
        const uint32_t full = mode == CUPBR_BATCH_COOPERATIVE
                                  ? (uint32_t)batch_coop_occupancy()
                                  : (uint32_t)batch_persistent_occupancy(pers_threads, pers_packets);
        return pers_blocks ? std::min(pers_blocks, full) : full;
    }
    // Tables both modes (and the adjoint) use: views, scene records, work
    // items heaviest first, the item counter.
    cudaError_t build_tables(const std::vector<BatchView>& table) {
        std::vector<uint32_t> nodes(scenes.size());
        std::vector<DeviceScene> ds(scenes.size());
        scene_gen.resize(scenes.size());
        for (size_t i = 0; i < scenes.size(); ++i) {
            ds[i] = scenes[i]->g.dev;
            nodes[i] = ds[i].n_nodes;
            scene_gen[i] = scenes[i]->g.generation;
        }
        std::vector<BatchItem> items;
        batch_items(table, nodes, items);
        n_items = (uint32_t)items.size();
        cudaError_t e;
        if ((e = dev_alloc(&dviews, sizeof(BatchView) * table.size())) != cudaSuccess) return e;
        if ((e = dev_alloc(&dscenes, sizeof(DeviceScene) * ds.size())) != cudaSuccess) return e;
        if ((e = dev_alloc(&ditems, sizeof(BatchItem) * std::max<size_t>(1, items.size()))) != cudaSuccess) return e;
        if ((e = dev_alloc(&dcounter, sizeof(uint32_t) * 2)) != cudaSuccess) return e;
        if ((e = cudaMemset(dcounter, 0, sizeof(uint32_t) * 2)) != cudaSuccess) return e;
        if ((e = cudaMemcpy(dviews, table.data(), sizeof(BatchView) * table.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return e;
        if ((e = cudaMemcpy(dscenes, ds.data(), sizeof(DeviceScene) * ds.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return e;
        if (!items.empty() &&
            (e = cudaMemcpy(ditems, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return e;
        return cudaSuccess;
    }
    // The persistent kernel's graph (counter reset + one launch).
    cudaError_t build_persistent() {
        cudaError_t e;
        if (!cap && (e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)) != cudaSuccess) return e;
        if ((e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
        const cudaError_t rec = batch_launch_persistent(dscenes, dviews, ditems, n_items, dcounter, max_depth,
                                                        pers_threads, blocks_per_sm(), pers_packets,
                                                        device_sm_count(), dcounter + 1, cap);
        e = cudaStreamEndCapture(cap, &graph);
        if (rec != cudaSuccess) return rec;
        if (e != cudaSuccess) return e;
        if ((e = cudaGraphInstantiate(&exec, graph, 0)) != cudaSuccess) return e;
        waves.clear();
        segs.clear();
        launches_per_replay = 1;
        dirty = false;
        return cudaSuccess;
    }
    uint32_t max_pixels() const {
        uint32_t m = 0;
        for (const BatchView& v : views) m = std::max(m, v.width * v.height);
        return m;
    }
    // Plans the wavefronts for the current views and settings, (re)allocates
    // the queues and tables, and captures the launch sequence as a graph.
    cudaError_t build(const std::vector<BatchView>& table) {
        release_graph();
        free_tables();
        cudaError_t et = build_tables(table);
        if (et != cudaSuccess) return et;
        if (mode == CUPBR_BATCH_PERSISTENT) return build_persistent();
        const uint32_t capacity = std::max(batch_paths, max_pixels());
        batch_plan(view_scene, table, (uint32_t)scenes.size(), capacity, waves, segs);
        uint32_t need = 0;
        for (const BatchWave& w : waves) need = std::max(need, w.n_paths);
        cudaError_t e = pt.ensure(need);
        if (e != cudaSuccess) return e;
        const int full = pt_occupancy_blocks((int)(pt.ws.smem_nodes * BVH_NODE_BYTES));
        pt.ws.trace_blocks_per_sm = std::max(1, (int)(full * trace_share + 0.5f));
        if ((e = dev_alloc(&dsegs, sizeof(BatchSegment) * std::max<size_t>(1, segs.size()))) != cudaSuccess) return e;
        if (!segs.empty() &&
            (e = cudaMemcpy(dsegs, segs.data(), sizeof(BatchSegment) * segs.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return e;
        const bool coop = mode == CUPBR_BATCH_COOPERATIVE;
        if (coop) {
            if ((e = dev_alloc(&dwaves, sizeof(BatchWave) * std::max<size_t>(1, waves.size()))) != cudaSuccess) return e;
            if ((e = dev_alloc(&dbar, sizeof(BatchBarrier))) != cudaSuccess) return e;
            if ((e = cudaMemset(dbar, 0, sizeof(BatchBarrier))) != cudaSuccess) return e;
            if (!waves.empty() &&
                (e = cudaMemcpy(dwaves, waves.data(), sizeof(BatchWave) * waves.size(), cudaMemcpyHostToDevice)) !=
                    cudaSuccess)
                return e;
        }
        if (!cap && (e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)) != cudaSuccess) return e;
        if ((e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
        cudaError_t rec = cudaSuccess;
        if (coop) {
            rec = batch_launch_coop(dscenes, dwaves, (uint32_t)waves.size(), dsegs, dviews, pt.ws, max_depth,
                                    blocks_per_sm(), device_sm_count(), dbar, cap, barrier_probe_ns);
        } else {
            for (const BatchWave& w : waves) {
                rec = batch_record_wave(scenes[w.scene]->g.dev, w, dsegs, dviews, pt.ws, max_depth, device_sm_count(),
                                        cap);
                if (rec != cudaSuccess) break;
            }
        }
        e = cudaStreamEndCapture(cap, &graph);
        if (rec != cudaSuccess) return rec;
        if (e != cudaSuccess) return e;
        if ((e = cudaGraphInstantiate(&exec, graph, 0)) != cudaSuccess) return e;
        launches_per_replay = coop ? 1u : (uint32_t)waves.size() * (2 + 3 * max_depth);
        dirty = false;
        return cudaSuccess;
    }
    // a scene re-committed since the build (another batch's autotuner rebuilt
    // its BVH) has new device buffers: the tables and graph are rebuilt
    bool scenes_changed() const {
        for (size_t i = 0; i < scenes.size(); ++i)
            if (i >= scene_gen.size() || scene_gen[i] != scenes[i]->g.generation) return true;
        return false;
    }
    cudaError_t launch(cudaStream_t st) {
        cudaError_t e;
        if (scenes_changed()) {
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
            if ((e = build(views)) != cudaSuccess) return e;
        }
        if (dirty) {
            if ((e = cudaMemcpyAsync(dviews, views.data(), sizeof(BatchView) * views.size(), cudaMemcpyHostToDevice,
                                     st)) != cudaSuccess)
                return e;
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;  // the host table may change again
            dirty = false;
        }
        return cudaGraphLaunch(exec, st);
    }
};

int cupbr_batch_create(const cupbr_view* views, uint32_t n_views, uint32_t max_depth, cupbr_batch_t* out) {
    if (!views || !out || n_views == 0) return fail(CUPBR_ERR_ARG, "no views");
    if (max_depth == 0 || max_depth > PT_MAX_DEPTH)
        return fail(CUPBR_ERR_ARG, "max_depth must lie in [1, " + std::to_string(PT_MAX_DEPTH) + "]");
    std::unique_ptr<cupbr_batch_s> b(new cupbr_batch_s());
    b->max_depth = max_depth;
    for (uint32_t i = 0; i < n_views; ++i) {
        const cupbr_view& v = views[i];
        if (!v.scene || !v.device_image) return fail(CUPBR_ERR_ARG, "view " + std::to_string(i) + ": null scene or image");
        if (!v.scene->g.committed) return fail(CUPBR_ERR_STATE, "view " + std::to_string(i) + ": scene not committed");
        if (v.width == 0 || v.height == 0 || v.spp == 0)
            return fail(CUPBR_ERR_ARG, "view " + std::to_string(i) + ": empty image or no samples");
        if ((uint64_t)v.width * v.height > (1u << 26))
            return fail(CUPBR_ERR_ARG, "view " + std::to_string(i) + ": image above 2^26 pixels");
        uint32_t si = 0;
        while (si < b->scenes.size() && b->scenes[si] != v.scene) ++si;
        if (si == b->scenes.size()) b->scenes.push_back(v.scene);
        b->view_scene.push_back(si);
        BatchView bv;
        const cupbr_camera& c = v.camera;
        bv.cam_pos = mk(c.position.x, c.position.y, c.position.z);
        bv.cam_x = mk(c.x_axis.x, c.x_axis.y, c.x_axis.z);
        bv.cam_y = mk(c.y_axis.x, c.y_axis.y, c.y_axis.z);
        bv.cam_z = mk(c.z_axis.x, c.z_axis.y, c.z_axis.z);
        bv.width = v.width;
        bv.height = v.height;
        bv.frame0 = v.frame0;
        bv.spp = v.spp;
        bv.img = v.device_image;
        bv.scene = si;
        b->views.push_back(bv);
    }
    CUPBR_CHECK_CUDA(b->build(b->views));
    *out = b.release();
    return CUPBR_OK;
}
int cupbr_batch_destroy(cupbr_batch_t b) {
    delete b;
    return CUPBR_OK;
}
int cupbr_batch_launch(cupbr_batch_t b, void* stream) {
    NvtxRange nvtx_("cupbr_batch_launch");
    if (!b) return fail(CUPBR_ERR_ARG, "null batch");
    CUPBR_CHECK_CUDA(b->launch((cudaStream_t)stream));
    return CUPBR_OK;
}
int cupbr_batch_advance(cupbr_batch_t b) {
    if (!b) return fail(CUPBR_ERR_ARG, "null batch");
    for (BatchView& v : b->views) v.frame0 += v.spp;
    b->dirty = true;
    return CUPBR_OK;
}
int cupbr_batch_set_frame0(cupbr_batch_t b, uint32_t view, uint32_t frame0) {
    if (!b || view >= b->views.size()) return fail(CUPBR_ERR_ARG, "view index out of range");
    b->views[view].frame0 = frame0;
    b->dirty = true;
    return CUPBR_OK;
}
int cupbr_batch_get_info(cupbr_batch_t b, uint32_t* wavefronts, uint64_t* paths, uint32_t* kernel_launches,
                         uint32_t* batch_paths) {
    if (!b) return fail(CUPBR_ERR_ARG, "null batch");
    uint64_t n = 0;
    for (const BatchView& v : b->views) n += (uint64_t)v.width * v.height * v.spp;
    if (wavefronts) *wavefronts = (uint32_t)b->waves.size();
    if (paths) *paths = n;
    if (kernel_launches) *kernel_launches = b->launches_per_replay;
    if (batch_paths) *batch_paths = b->batch_paths;
    return CUPBR_OK;
}
int cupbr_batch_configure(cupbr_batch_t b, uint32_t batch_paths, float trace_share) {
    if (!b || batch_paths == 0 || !(trace_share > 0.0f && trace_share <= 1.0f))
        return fail(CUPBR_ERR_ARG, "batch_paths >= 1 and 0 < trace_share <= 1 required");
    b->batch_paths = batch_paths;
    b->trace_share = trace_share;
    CUPBR_CHECK_CUDA(b->build(b->views));
    return CUPBR_OK;
}
int cupbr_batch_set_mode(cupbr_batch_t b, int32_t mode, uint32_t threads_per_block, uint32_t blocks_per_sm,
                         int32_t camera_packets) {
    if (!b) return fail(CUPBR_ERR_ARG, "null batch");
    if (mode != CUPBR_BATCH_WAVEFRONT && mode != CUPBR_BATCH_PERSISTENT && mode != CUPBR_BATCH_COOPERATIVE)
        return fail(CUPBR_ERR_ARG, "unknown batch mode");
    if (threads_per_block != 64 && threads_per_block != 128 && threads_per_block != 256)
        return fail(CUPBR_ERR_ARG, "threads_per_block must be 64, 128 or 256");
    if (mode == CUPBR_BATCH_COOPERATIVE && threads_per_block != 256)
        return fail(CUPBR_ERR_ARG, "the cooperative kernel runs 256 threads per block");
    b->mode = mode;
    b->pers_threads = threads_per_block;
    b->pers_blocks = blocks_per_sm;
    b->pers_packets = camera_packets != 0;
    CUPBR_CHECK_CUDA(b->build(b->views));
    return CUPBR_OK;
}
int cupbr_batch_get_mode(cupbr_batch_t b, int32_t* mode, uint32_t* threads_per_block, uint32_t* blocks_per_sm,
                         int32_t* camera_packets) {
    if (!b) return fail(CUPBR_ERR_ARG, "null batch");
    if (mode) *mode = b->mode;
    if (threads_per_block) *threads_per_block = b->pers_threads;
    if (blocks_per_sm) *blocks_per_sm = b->mode != CUPBR_BATCH_WAVEFRONT ? b->blocks_per_sm() : 0u;
    if (camera_packets) *camera_packets = b->pers_packets ? 1 : 0;
    return CUPBR_OK;
}
int cupbr_batch_set_barrier_probe(cupbr_batch_t b, uint64_t ns) {
    if (!b) return fail(CUPBR_ERR_ARG, "null batch");
    if (ns > 1000000000ull) return fail(CUPBR_ERR_ARG, "probe limit above 1 s");
    b->barrier_probe_ns = ns;
    if (b->mode == CUPBR_BATCH_COOPERATIVE) CUPBR_CHECK_CUDA(b->build(b->views));
    return CUPBR_OK;
}
int cupbr_batch_get_error_count(cupbr_batch_t b, uint32_t* out) {
    if (!b || !out) return fail(CUPBR_ERR_ARG, "null argument");
    CUPBR_CHECK_CUDA(cudaDeviceSynchronize());
    *out = 0;
    if (b->dcounter) CUPBR_CHECK_CUDA(cudaMemcpy(out, b->dcounter + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (b->pt.ws.err) {
        uint32_t e[ERR_TOTAL];
        CUPBR_CHECK_CUDA(cudaMemcpy(e, b->pt.ws.err, sizeof e, cudaMemcpyDeviceToHost));
        for (uint32_t k = 0; k < ERR_TOTAL; ++k) *out += e[k];
    }
    if (b->dbar) {
        BatchBarrier gb;
        CUPBR_CHECK_CUDA(cudaMemcpy(&gb, b->dbar, sizeof gb, cudaMemcpyDeviceToHost));
        *out += gb.abort;
    }
    return CUPBR_OK;
}

int cupbr_batch_backward(cupbr_batch_t b, const uint64_t* device_grad_images, int32_t accumulate, void* stream) {
    NvtxRange nvtx_("cupbr_batch_backward");
    if (!b || !device_grad_images) return fail(CUPBR_ERR_ARG, "null argument");
    if (b->max_depth > BATCH_BWD_MAX_DEPTH)
        return fail(CUPBR_ERR_ARG, "the texture adjoint records at most " + std::to_string(BATCH_BWD_MAX_DEPTH) +
                                       " vertices per path: max_depth too large");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nv = b->views.size(), ns = b->scenes.size();
    b->tex_grad.resize(ns, nullptr);
    bool any = false;
    for (size_t i = 0; i < ns; ++i) {
        const DeviceScene& d = b->scenes[i]->g.dev;
        if (!d.tex) continue;
        any = true;
        const size_t bytes = sizeof(float) * 3 * (size_t)d.tex_w * d.tex_h;
        if (!b->tex_grad[i]) {
            CUPBR_CHECK_CUDA(dev_alloc(&b->tex_grad[i], bytes));
            CUPBR_CHECK_CUDA(cudaMemsetAsync(b->tex_grad[i], 0, bytes, st));
        } else if (!accumulate) {
            CUPBR_CHECK_CUDA(cudaMemsetAsync(b->tex_grad[i], 0, bytes, st));
        }
    }
    if (!any) return fail(CUPBR_ERR_STATE, "no scene of the batch has an albedo texture");
    if (b->scenes_changed()) {
        CUPBR_CHECK_CUDA(cudaStreamSynchronize(st));
        CUPBR_CHECK_CUDA(b->build(b->views));
    }
    if (!b->dgrad_img) CUPBR_CHECK_CUDA(dev_alloc(&b->dgrad_img, sizeof(float*) * nv));
    if (!b->dgrad_tex) CUPBR_CHECK_CUDA(dev_alloc(&b->dgrad_tex, sizeof(float*) * ns));
    std::vector<const float*> gi(nv);
    for (size_t i = 0; i < nv; ++i) gi[i] = reinterpret_cast<const float*>(device_grad_images[i]);
    CUPBR_CHECK_CUDA(cudaMemcpyAsync(b->dgrad_img, gi.data(), sizeof(float*) * nv, cudaMemcpyHostToDevice, st));
    CUPBR_CHECK_CUDA(cudaMemcpyAsync(b->dgrad_tex, b->tex_grad.data(), sizeof(float*) * ns, cudaMemcpyHostToDevice, st));
    if (b->dirty) {
        CUPBR_CHECK_CUDA(cudaMemcpyAsync(b->dviews, b->views.data(), sizeof(BatchView) * nv, cudaMemcpyHostToDevice, st));
        b->dirty = false;
    }
    const uint32_t threads = b->pers_threads;
    const uint32_t blocks = (uint32_t)batch_backward_occupancy(threads);
    CUPBR_CHECK_CUDA(batch_launch_backward(b->dscenes, b->dviews, b->ditems, b->n_items, b->dcounter, b->max_depth,
                                           b->dgrad_img, b->dgrad_tex, threads, blocks, device_sm_count(),
                                           b->dcounter + 1, st));
    // the host tables above are pageable: the copies are done when the calls return
    CUPBR_CHECK_CUDA(cudaStreamSynchronize(st));
    return CUPBR_OK;
}
int cupbr_batch_get_texture_gradient(cupbr_batch_t b, cupbr_scene_t scene, float** device_grad_rgb, uint32_t* w,
                                     uint32_t* h) {
    if (!b || !scene || !device_grad_rgb) return fail(CUPBR_ERR_ARG, "null argument");
    for (size_t i = 0; i < b->scenes.size(); ++i)
        if (b->scenes[i] == scene) {
            *device_grad_rgb = i < b->tex_grad.size() ? b->tex_grad[i] : nullptr;
            if (w) *w = scene->g.dev.tex_w;
            if (h) *h = scene->g.dev.tex_h;
            return CUPBR_OK;
        }
    return fail(CUPBR_ERR_ARG, "scene not in this batch");
}

namespace {

// One candidate configuration of a batch.
struct BatchCand {
    int32_t mode;
    uint32_t threads, blocks;  // persistent
    bool packets;              // persistent: camera rays as warp packets
    uint32_t size;             // wavefront
    float share;               // wavefront
    int leaf;                  // BVH leaf size of every scene (0: as committed)
};

}  // namespace

int cupbr_batch_autotune_ex(cupbr_batch_t b, void* stream, uint32_t flags, float* best_ms) {
    NvtxRange nvtx_("cupbr_batch_autotune_ex");
    if (!b) return fail(CUPBR_ERR_ARG, "null batch");
    if (flags & ~CUPBR_TUNE_BVH_LEAF) return fail(CUPBR_ERR_ARG, "unknown autotune flag");
    cudaStream_t st = (cudaStream_t)stream;
    // scratch images, so tuning leaves the views' running means alone
    size_t floats = 0;
    for (const BatchView& v : b->views) floats += 3 * (size_t)v.width * v.height;
    float* scratch = nullptr;
    CUPBR_CHECK_CUDA(dev_alloc(&scratch, sizeof(float) * floats));
    std::vector<BatchView> table = b->views;
    size_t off = 0;
    for (BatchView& v : table) {
        v.img = scratch + off;
        off += 3 * (size_t)v.width * v.height;
    }
    std::vector<BvhBuildParams> committed;
    for (cupbr_scene_s* sc : b->scenes) committed.push_back(sc->g.params);
    // (re)commits every scene with leaf size `leaf` (0: as committed)
    int cur_leaf = 0;
    auto set_leaf = [&](int leaf) -> bool {
        if (leaf == cur_leaf) return true;
        for (size_t i = 0; i < b->scenes.size(); ++i) {
            BvhBuildParams p = committed[i];
            if (leaf) p.max_leaf = leaf;
            std::string why;
            if (!commit_scene(b->scenes[i]->g, p, why)) return false;
        }
        cur_leaf = leaf;
        return true;
    };
    // first the persistent kernel at 128 threads and full occupancy with and
    // without camera packets, and wavefronts of 2^21..2^25 paths at full
    // traversal occupancy; then, around the best of those, the persistent
    // kernel's other block shapes (64 and 256 threads, half occupancy) or
    // the best wavefront size at 3/4 occupancy; then the best configuration
    // at leaf sizes 2 and 8 (CUPBR_TUNE_BVH_LEAF)
    std::vector<BatchCand> cands;
    for (bool pk : {true, false}) {
        const uint32_t full = (uint32_t)batch_persistent_occupancy(128, pk);
        cands.push_back({CUPBR_BATCH_PERSISTENT, 128, full, pk, 0, 1.0f, 0});
    }
    for (uint32_t sz = 1u << 21; sz <= 1u << 25; sz <<= 1)
        cands.push_back({CUPBR_BATCH_WAVEFRONT, 128, 0, true, sz, 1.0f, 0});
    for (uint32_t sz : {1u << 22, 1u << 24})
        cands.push_back({CUPBR_BATCH_COOPERATIVE, 256, 0, true, sz, 1.0f, 0});
    const size_t n_first = cands.size();
    size_t n_second = 0;
    float best = 1e30f;
    BatchCand best_c{b->mode, b->pers_threads, b->pers_blocks, b->pers_packets, b->batch_paths, b->trace_share, 0};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaEventCreate(&e0);
    if (err == cudaSuccess) err = cudaEventCreate(&e1);
    bool commit_failed = false;
    for (size_t k = 0; k < cands.size() && err == cudaSuccess; ++k) {
        const BatchCand& c = cands[k];
        if (!set_leaf(c.leaf)) { commit_failed = true; break; }
        b->mode = c.mode;
        b->pers_threads = c.threads;
        b->pers_blocks = c.blocks;
        b->pers_packets = c.packets;
        if (c.mode != CUPBR_BATCH_PERSISTENT) {
            b->batch_paths = c.size;
            b->trace_share = c.share;
        }
        if ((err = b->build(table)) != cudaSuccess) break;
        // the median of three timed replays
        float t[3];
        for (int r = 0; r < 3 && err == cudaSuccess; ++r) {
            cudaEventRecord(e0, st);
            if ((err = cudaGraphLaunch(b->exec, st)) != cudaSuccess) break;
            cudaEventRecord(e1, st);
            if ((err = cudaEventSynchronize(e1)) != cudaSuccess) break;
            cudaEventElapsedTime(&t[r], e0, e1);
        }
        if (err != cudaSuccess) break;
        std::sort(t, t + 3);
        if (t[1] < best) {
            best = t[1];
            best_c = c;
        }
        if (k + 1 == n_first) {
            const BatchCand c2 = best_c;
            if (c2.mode == CUPBR_BATCH_WAVEFRONT) {
                BatchCand c3 = c2;
                c3.share = 0.75f;
                cands.push_back(c3);
            } else if (c2.mode == CUPBR_BATCH_COOPERATIVE) {
                for (uint32_t sz : {c2.size / 2, c2.size * 2}) {
                    BatchCand c3 = c2;
                    c3.size = sz;
                    cands.push_back(c3);
                }
            } else {
                for (uint32_t t : {64u, 256u}) {
                    BatchCand c3 = c2;
                    c3.threads = t;
                    c3.blocks = (uint32_t)batch_persistent_occupancy(t, c2.packets);
                    cands.push_back(c3);
                }
                BatchCand c3 = c2;
                c3.blocks = std::max(1u, c2.blocks / 2);
                cands.push_back(c3);
            }
            n_second = cands.size();
        } else if (k + 1 == n_second && (flags & CUPBR_TUNE_BVH_LEAF)) {
            for (int leaf : {2, 8}) {
                BatchCand cl = best_c;
                cl.leaf = leaf;
                cands.push_back(cl);
            }
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamSynchronize(st);
    cudaFree(scratch);
    if (err != cudaSuccess) return cuda_fail(err, "batch autotune");
    if (commit_failed || !set_leaf(best_c.leaf)) return fail(CUPBR_ERR_CUDA, "batch autotune: scene re-commit failed");
    b->mode = best_c.mode;
    b->pers_threads = best_c.threads;
    b->pers_blocks = best_c.blocks;
    b->pers_packets = best_c.packets;
    if (best_c.mode != CUPBR_BATCH_PERSISTENT) {
        b->batch_paths = best_c.size;
        b->trace_share = best_c.share;
    }
    CUPBR_CHECK_CUDA(b->build(b->views));
    if (best_ms) *best_ms = best;
    return CUPBR_OK;
}
int cupbr_batch_autotune(cupbr_batch_t b, void* stream, float* best_ms) {
    return cupbr_batch_autotune_ex(b, stream, 0u, best_ms);
}

// ------------------------------------------------------------ helpers ---
// ------------------------------------------------------ radiance cache ---
struct cupbr_cache_s {
    cupbr_cache_desc desc{};
    RcNet net;
    RcBounds bounds{};
    uint32_t step = 0;  // Adam steps taken
    PTBuffers pt;
    std::vector<void*> bufs;
    float4* queries = nullptr;
    uint32_t* counters = nullptr;  // [0] queries, [1] samples
    float4* tverts = nullptr;
    uint32_t* tcount = nullptr;
    uint32_t path_capacity = 0, depth_capacity = 0, train_capacity = 0;
    float4* samples = nullptr;
    uint32_t sample_capacity = 0;
    uint32_t batch_paths = 1u << 25;  // paths per wavefront (whole frames, at least one)
    uint32_t tail_paths = 1u << 16;   // ray queues below this go to the per-path tail kernel
    bool profiling = false;
    // set once a CTA freed its tensor memory with MMAs possibly still in
    // flight (err[1] > 0): the network state can no longer be trusted
    bool lost = false;
    // profiled wavefronts: events [0] start, [1] after the camera kernel, 3 per
    // depth (after extend / shade / connect), then after inference, after
    // accumulation + sample collection, after training
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::vector<cudaEvent_t>> ev_frames;
    ~cupbr_cache_s() {
        for (void* p : bufs) cudaFree(p);
        for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
        for (auto& f : ev_frames)
            for (cudaEvent_t e : f) cudaEventDestroy(e);
    }
    cudaError_t take_events(size_t n, std::vector<cudaEvent_t>& out) {
        out.clear();
        while (out.size() < n) {
            if (ev_pool.empty()) {
                cudaEvent_t e;
                cudaError_t err = cudaEventCreate(&e);
                if (err != cudaSuccess) return err;
                ev_pool.push_back(e);
            }
            out.push_back(ev_pool.back());
            ev_pool.pop_back();
        }
        return cudaSuccess;
    }
    cudaError_t alloc(void** p, size_t bytes) {
        cudaError_t e = dev_alloc(p, bytes);
        if (e == cudaSuccess) bufs.push_back(*p);
        return e;
    }
    void drop(void* p) {
        if (!p) return;
        for (auto& b : bufs)
            if (b == p) {
                cudaFree(b);
                b = bufs.back();
                bufs.pop_back();
                break;
            }
    }
    // queries / training-vertex buffers for n paths of depth max_depth
    cudaError_t ensure(uint32_t n, uint32_t depth) {
        cudaError_t e = pt.ensure(n);
        if (e != cudaSuccess) return e;
        if (n > path_capacity) {
            drop(queries);
            queries = nullptr;
            path_capacity = 0;
            if ((e = alloc((void**)&queries, sizeof(float4) * RC_REC * (size_t)n)) != cudaSuccess) return e;
            path_capacity = n;
        }
        // training paths: one per train_stride paths (one slot when training is off)
        const uint32_t ntrain = desc.train_stride ? (path_capacity + desc.train_stride - 1) / desc.train_stride : 1u;
        if (depth > depth_capacity || ntrain > train_capacity) {
            drop(tverts);
            drop(tcount);
            tverts = nullptr;
            tcount = nullptr;
            depth_capacity = train_capacity = 0;
            const uint32_t d = std::max(depth, 8u);
            if ((e = alloc((void**)&tverts, sizeof(float4) * RC_REC * (size_t)ntrain * d)) != cudaSuccess) return e;
            if ((e = alloc((void**)&tcount, sizeof(uint32_t) * (size_t)ntrain)) != cudaSuccess) return e;
            depth_capacity = d;
            train_capacity = ntrain;
        }
        return cudaSuccess;
    }
    RcAdam adam() { return RcAdam{desc.learning_rate, 0.9f, 0.99f, 1e-15f, ++step, desc.weight_average, desc.loss}; }
    // inference weights: the bias-corrected weight average once training has stepped
    const __half* infer_weights() const { return desc.weight_average > 0.0f && step > 0 ? net.w16_ema : net.w16; }
};

namespace {

uint64_t rc_splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// parameter index (layer-major, row-major [out][in], 3 output rows) ->
// tiled weight index
void rc_param_map(std::vector<uint32_t>& tiled_of_param) {
    tiled_of_param.clear();
    for (uint32_t l = 0; l < RC_LAYERS; ++l) {
        const uint32_t rows = l + 1 == RC_LAYERS ? 3u : rc_out(l), K = rc_in(l);
        for (uint32_t o = 0; o < rows; ++o)
            for (uint32_t i = 0; i < K; ++i) tiled_of_param.push_back(rc_woff(l) + rc_tiled(o, i, K));
    }
}

cudaError_t rc_upload(cupbr_cache_s* c, const std::vector<float>& tiled) {
    std::vector<__half> h(RC_WEIGHTS);
    for (uint32_t i = 0; i < RC_WEIGHTS; ++i) h[i] = __float2half_rn(tiled[i]);
    cudaError_t e;
    if ((e = cudaMemcpy(c->net.master, tiled.data(), sizeof(float) * RC_WEIGHTS, cudaMemcpyHostToDevice)) !=
        cudaSuccess)
        return e;
    if ((e = cudaMemcpy(c->net.w16, h.data(), sizeof(__half) * RC_WEIGHTS, cudaMemcpyHostToDevice)) != cudaSuccess)
        return e;
    if ((e = cudaMemset(c->net.adam_m, 0, sizeof(float) * RC_WEIGHTS)) != cudaSuccess) return e;
    if ((e = cudaMemset(c->net.adam_v, 0, sizeof(float) * RC_WEIGHTS)) != cudaSuccess) return e;
    if ((e = cudaMemset(c->net.ema, 0, sizeof(float) * RC_WEIGHTS)) != cudaSuccess) return e;
    c->step = 0;
    return cudaSuccess;
}

}  // namespace

int cupbr_cache_create(cupbr_scene_t s, const cupbr_cache_desc* desc, cupbr_cache_t* out) {
    if (!s || !desc || !out) return fail(CUPBR_ERR_ARG, "null argument");
    if (!s->g.committed) return fail(CUPBR_ERR_STATE, "scene not committed");
    cupbr_cache_desc d = *desc;
    if (d.batch == 0) d.batch = 1u << 14;
    if (d.samples_per_frame == 0) d.samples_per_frame = 1u << 16;
    if (!(d.learning_rate > 0.0f)) d.learning_rate = 1e-2f;
    if (d.batch % RC_TILE != 0 || d.batch > (1u << 20))
        return fail(CUPBR_ERR_ARG, "batch must be a multiple of 128, at most 2^20");
    if (d.samples_per_frame % d.batch != 0) return fail(CUPBR_ERR_ARG, "samples_per_frame must be a multiple of batch");
    if (d.cache_depth >= PT_MAX_DEPTH) return fail(CUPBR_ERR_ARG, "cache_depth out of range");
    if (d.loss > RC_LOSS_L2) return fail(CUPBR_ERR_ARG, "unknown loss");
    if (d.train_suffix >= PT_MAX_DEPTH) return fail(CUPBR_ERR_ARG, "train_suffix out of range");
    if (!(d.weight_average >= 0.0f && d.weight_average < 1.0f)) return fail(CUPBR_ERR_ARG, "weight_average must be in [0, 1)");
    std::unique_ptr<cupbr_cache_s> c(new cupbr_cache_s());
    c->desc = d;
    RcNet& N = c->net;
    N.partial_ctas = d.batch / RC_TILE;
    CUPBR_CHECK_CUDA(c->alloc((void**)&N.master, sizeof(float) * RC_WEIGHTS));
    CUPBR_CHECK_CUDA(c->alloc((void**)&N.adam_m, sizeof(float) * RC_WEIGHTS));
    CUPBR_CHECK_CUDA(c->alloc((void**)&N.adam_v, sizeof(float) * RC_WEIGHTS));
    CUPBR_CHECK_CUDA(c->alloc((void**)&N.grad, sizeof(float) * RC_WEIGHTS));
    CUPBR_CHECK_CUDA(c->alloc((void**)&N.w16, sizeof(__half) * RC_WEIGHTS));
    CUPBR_CHECK_CUDA(c->alloc((void**)&N.ema, sizeof(float) * RC_WEIGHTS));
    CUPBR_CHECK_CUDA(c->alloc((void**)&N.w16_ema, sizeof(__half) * RC_WEIGHTS));
    CUPBR_CHECK_CUDA(c->alloc((void**)&N.partials, sizeof(float) * RC_WEIGHTS * (size_t)N.partial_ctas));
    CUPBR_CHECK_CUDA(c->alloc((void**)&N.loss, sizeof(float) * 2));
    CUPBR_CHECK_CUDA(c->alloc((void**)&N.err, sizeof(uint32_t) * 2));
    CUPBR_CHECK_CUDA(c->alloc((void**)&c->counters, sizeof(uint32_t) * 2));
    CUPBR_CHECK_CUDA(cudaMemset(N.err, 0, sizeof(uint32_t) * 2));
    CUPBR_CHECK_CUDA(cudaMemset(N.grad, 0, sizeof(float) * RC_WEIGHTS));
    CUPBR_CHECK_CUDA(cudaMemset(N.loss, 0, sizeof(float) * 2));
    CUPBR_CHECK_CUDA(cudaMemset(c->counters, 0, sizeof(uint32_t) * 2));
    // He-uniform hidden layers, smaller output layer; unused output rows stay 0
    std::vector<float> w(RC_WEIGHTS, 0.0f);
    uint64_t rs = 0x5EEDull ^ ((uint64_t)d.seed << 20);
    for (uint32_t l = 0; l < RC_LAYERS; ++l) {
        const bool last = l + 1 == RC_LAYERS;
        const uint32_t rows = last ? 3u : rc_out(l), K = rc_in(l);
        const float a = last ? std::sqrt(1.0f / (float)K) : std::sqrt(6.0f / (float)K);
        for (uint32_t o = 0; o < rows; ++o)
            for (uint32_t i = 0; i < K; ++i) {
                const double u = (double)(rc_splitmix(rs) >> 11) * (1.0 / 9007199254740992.0);
                w[rc_woff(l) + rc_tiled(o, i, K)] = (float)((2.0 * u - 1.0) * a);
            }
    }
    CUPBR_CHECK_CUDA(rc_upload(c.get(), w));
    // position box: union of the root node's children
    const std::vector<float>& nodes = s->g.bvh.nodes;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (nodes.size() >= 32) {
        for (int k = 0; k < 4; ++k) {
            int32_t ref;
            std::memcpy(&ref, &nodes[24 + k], 4);
            if (ref == BVH_EMPTY) continue;
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], nodes[8 * a + k]);
                hi[a] = std::max(hi[a], nodes[8 * a + 4 + k]);
            }
        }
    }
    float l3[3], inv[3];
    for (int a = 0; a < 3; ++a) {
        if (!(hi[a] >= lo[a]) || !std::isfinite(lo[a]) || !std::isfinite(hi[a])) {
            lo[a] = -1.0f;
            hi[a] = 1.0f;
        }
        const float ext = std::max(hi[a] - lo[a], 1e-6f);
        l3[a] = lo[a];
        inv[a] = 1.0f / ext;
    }
    c->bounds.lo = mk(l3[0], l3[1], l3[2]);
    c->bounds.inv_ext = mk(inv[0], inv[1], inv[2]);
    *out = c.release();
    return CUPBR_OK;
}
int cupbr_cache_destroy(cupbr_cache_t c) {
    delete c;
    return CUPBR_OK;
}
uint32_t cupbr_cache_param_count(void) { return RC_PARAMS; }
int cupbr_cache_get_bounds(cupbr_cache_t c, float* lo, float* inv) {
    if (!c || !lo || !inv) return fail(CUPBR_ERR_ARG, "null argument");
    lo[0] = c->bounds.lo.x;
    lo[1] = c->bounds.lo.y;
    lo[2] = c->bounds.lo.z;
    inv[0] = c->bounds.inv_ext.x;
    inv[1] = c->bounds.inv_ext.y;
    inv[2] = c->bounds.inv_ext.z;
    return CUPBR_OK;
}
int cupbr_cache_get_params(cupbr_cache_t c, float* host) {
    if (!c || !host) return fail(CUPBR_ERR_ARG, "null argument");
    CUPBR_CHECK_CUDA(cudaDeviceSynchronize());
    std::vector<float> t(RC_WEIGHTS);
    CUPBR_CHECK_CUDA(cudaMemcpy(t.data(), c->net.master, sizeof(float) * RC_WEIGHTS, cudaMemcpyDeviceToHost));
    std::vector<uint32_t> map;
    rc_param_map(map);
    for (size_t i = 0; i < map.size(); ++i) host[i] = t[map[i]];
    return CUPBR_OK;
}
int cupbr_cache_set_params(cupbr_cache_t c, const float* host) {
    if (!c || !host) return fail(CUPBR_ERR_ARG, "null argument");
    std::vector<float> t(RC_WEIGHTS, 0.0f);
    std::vector<uint32_t> map;
    rc_param_map(map);
    for (size_t i = 0; i < map.size(); ++i) {
        if (!std::isfinite(host[i])) return fail(CUPBR_ERR_ARG, "non-finite parameter");
        t[map[i]] = host[i];
    }
    CUPBR_CHECK_CUDA(cudaDeviceSynchronize());
    CUPBR_CHECK_CUDA(rc_upload(c, t));
    return CUPBR_OK;
}
int cupbr_cache_save(cupbr_cache_t c, const char* path) {
    if (!c || !path) return fail(CUPBR_ERR_ARG, "null argument");
    std::vector<float> buf(4 * (size_t)RC_WEIGHTS);
    CUPBR_CHECK_CUDA(cudaDeviceSynchronize());
    float* const src[4] = {c->net.master, c->net.adam_m, c->net.adam_v, c->net.ema};
    for (int k = 0; k < 4; ++k)
        CUPBR_CHECK_CUDA(cudaMemcpy(buf.data() + (size_t)k * RC_WEIGHTS, src[k], sizeof(float) * RC_WEIGHTS,
                                    cudaMemcpyDeviceToHost));
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(CUPBR_ERR_IO, std::string("cannot write ") + path);
    const uint32_t head[4] = {0x43425243u /* "CRBC" */, 2u, RC_WEIGHTS, c->step};
    bool ok = std::fwrite(head, sizeof(head), 1, f) == 1 &&
              std::fwrite(buf.data(), sizeof(float), buf.size(), f) == buf.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? CUPBR_OK : fail(CUPBR_ERR_IO, std::string("short write to ") + path);
}
int cupbr_cache_load(cupbr_cache_t c, const char* path) {
    if (!c || !path) return fail(CUPBR_ERR_ARG, "null argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(CUPBR_ERR_IO, std::string("cannot read ") + path);
    uint32_t head[4] = {0, 0, 0, 0};
    std::vector<float> buf(4 * (size_t)RC_WEIGHTS);
    bool ok = std::fread(head, sizeof(head), 1, f) == 1 && head[0] == 0x43425243u && head[1] == 2u &&
              head[2] == RC_WEIGHTS && std::fread(buf.data(), sizeof(float), buf.size(), f) == buf.size();
    std::fclose(f);
    if (!ok) return fail(CUPBR_ERR_IO, std::string("not a radiance-cache file: ") + path);
    CUPBR_CHECK_CUDA(cudaDeviceSynchronize());
    std::vector<float> master(buf.begin(), buf.begin() + RC_WEIGHTS);
    CUPBR_CHECK_CUDA(rc_upload(c, master));
    float* const dst[3] = {c->net.adam_m, c->net.adam_v, c->net.ema};
    for (int k = 0; k < 3; ++k)
        CUPBR_CHECK_CUDA(cudaMemcpy(dst[k], buf.data() + (size_t)(k + 1) * RC_WEIGHTS, sizeof(float) * RC_WEIGHTS,
                                    cudaMemcpyHostToDevice));
    c->step = head[3];
    // the inference copy of the weight average (bias-corrected)
    if (c->desc.weight_average > 0.0f && c->step > 0) {
        const double c3 = 1.0 - std::pow((double)c->desc.weight_average, (double)c->step);
        std::vector<__half> h(RC_WEIGHTS);
        for (uint32_t i = 0; i < RC_WEIGHTS; ++i)
            h[i] = __float2half_rn((float)(buf[3 * (size_t)RC_WEIGHTS + i] / c3));
        CUPBR_CHECK_CUDA(cudaMemcpy(c->net.w16_ema, h.data(), sizeof(__half) * RC_WEIGHTS, cudaMemcpyHostToDevice));
    }
    return CUPBR_OK;
}
static const char* const kCacheLost =
    "a tensor-core wait of this cache ran out twice and its tensor memory was freed with MMAs possibly in "
    "flight; destroy the cache";

int cupbr_cache_infer(cupbr_cache_t c, const float* recs, uint32_t n, float* out, void* stream) {
    if (!c || (n && (!recs || !out))) return fail(CUPBR_ERR_ARG, "null argument");
    if (c->lost) return fail(CUPBR_ERR_STATE, kCacheLost);
    CUPBR_CHECK_CUDA(rc_infer(c->net, c->infer_weights(), c->bounds, (const float4*)recs, n, (float4*)out,
                              device_sm_count(), (cudaStream_t)stream));
    return CUPBR_OK;
}
int cupbr_cache_train_step(cupbr_cache_t c, const float* samples, uint32_t n, void* stream) {
    if (!c || !samples) return fail(CUPBR_ERR_ARG, "null argument");
    if (c->lost) return fail(CUPBR_ERR_STATE, kCacheLost);
    if (n == 0 || n % RC_TILE != 0 || n / RC_TILE > c->net.partial_ctas)
        return fail(CUPBR_ERR_ARG, "n must be a positive multiple of 128, at most the batch size");
    CUPBR_CHECK_CUDA(rc_train_step(c->net, c->bounds, (const float4*)samples, nullptr, 0, 0, n, n, c->adam(),
                                   (cudaStream_t)stream));
    return CUPBR_OK;
}
int cupbr_cache_get_gradient(cupbr_cache_t c, float* host) {
    if (!c || !host) return fail(CUPBR_ERR_ARG, "null argument");
    CUPBR_CHECK_CUDA(cudaDeviceSynchronize());
    std::vector<float> t(RC_WEIGHTS);
    CUPBR_CHECK_CUDA(cudaMemcpy(t.data(), c->net.grad, sizeof(float) * RC_WEIGHTS, cudaMemcpyDeviceToHost));
    std::vector<uint32_t> map;
    rc_param_map(map);
    for (size_t i = 0; i < map.size(); ++i) host[i] = t[map[i]];
    return CUPBR_OK;
}
int cupbr_cache_get_loss(cupbr_cache_t c, float* loss, float* weighted) {
    if (!c || !loss) return fail(CUPBR_ERR_ARG, "null argument");
    CUPBR_CHECK_CUDA(cudaDeviceSynchronize());
    float l[2];
    CUPBR_CHECK_CUDA(cudaMemcpy(l, c->net.loss, sizeof(l), cudaMemcpyDeviceToHost));
    *loss = l[0] / (3.0f * std::max(l[1], 1.0f));
    if (weighted) *weighted = l[1];
    return CUPBR_OK;
}
int cupbr_cache_render(cupbr_cache_t c, cupbr_scene_t s, const cupbr_camera* cam, uint32_t w, uint32_t h,
                       uint32_t frame0, uint32_t frames, uint32_t depth, int32_t train, float* img, void* stream) {
    NvtxRange nvtx_("cupbr_cache_render");
    if (!c || !s || !cam || !img) return fail(CUPBR_ERR_ARG, "null argument");
    if (c->lost) return fail(CUPBR_ERR_STATE, kCacheLost);
    if (!s->g.committed) return fail(CUPBR_ERR_STATE, "scene not committed");
    if (w == 0 || h == 0 || (uint64_t)w * h >= (1ull << 30)) return fail(CUPBR_ERR_ARG, "bad image size");
    if (depth == 0 || depth > PT_MAX_DEPTH) return fail(CUPBR_ERR_ARG, "max trace depth must be 1..64");
    const cudaStream_t st = (cudaStream_t)stream;
    const int sms = device_sm_count();
    // several frames per wavefront (like cupbr_renderer_render_frames) up to batch_paths
    const uint32_t pixels = w * h;
    const uint32_t per_wave = std::max(1u, std::min(frames, c->batch_paths / pixels));
    CUPBR_CHECK_CUDA(c->ensure(pixels * per_wave, depth));
    const Workspace& W = c->pt.ws;
    const uint32_t stride = train ? c->desc.train_stride : 0u;
    const uint32_t steps_per_frame = c->desc.samples_per_frame / c->desc.batch;
    const uint32_t ntrain = stride ? (pixels * per_wave + stride - 1) / stride : 0u;
    const uint32_t want_samples = ntrain * depth;
    if (stride && c->sample_capacity < want_samples) {
        c->drop(c->samples);
        c->samples = nullptr;
        c->sample_capacity = 0;
        CUPBR_CHECK_CUDA(c->alloc((void**)&c->samples, sizeof(float4) * RC_REC * (size_t)want_samples));
        c->sample_capacity = want_samples;
    }
    for (uint32_t f = 0; f < frames;) {
        const uint32_t frame = frame0 + f;
        const uint32_t nf = std::min(per_wave, frames - f);
        f += nf;
        const uint32_t steps = steps_per_frame * nf;
        PTFrame F = make_frame(cam, w, h, frame, depth, false);
        F.frames = nf;
        F.n_paths = pixels * nf;
        CacheFrame C{};
        C.queries = c->queries;
        C.query_stride = F.n_paths;
        C.n_queries = c->counters;
        C.tverts = c->tverts;
        C.tcount = c->tcount;
        C.cache_depth = c->desc.cache_depth;
        C.specular = c->desc.cache_specular;
        C.train_end = c->desc.train_suffix ? c->desc.cache_depth + c->desc.train_suffix : 0u;
        C.tail_threshold = c->tail_paths;
        C.train_stride = stride;
        C.train_phase = stride ? (uint32_t)(((uint64_t)frame * 2654435761ull) >> 8) % stride : 0u;
        std::vector<cudaEvent_t> ev;
        size_t ei = 0;
        if (c->profiling) CUPBR_CHECK_CUDA(c->take_events(5 + 3 * (size_t)depth, ev));
        auto mark = [&]() -> cudaError_t { return c->profiling ? cudaEventRecord(ev[ei++], st) : cudaSuccess; };
        CUPBR_CHECK_CUDA(mark());
        CUPBR_CHECK_CUDA(cudaMemsetAsync(W.ctr, 0, sizeof(uint32_t) * CTR_TOTAL, st));
        CUPBR_CHECK_CUDA(cudaMemsetAsync(c->counters, 0, sizeof(uint32_t) * 2, st));
        if (stride) CUPBR_CHECK_CUDA(cudaMemsetAsync(c->tcount, 0, sizeof(uint32_t) * (size_t)ntrain, st));
        CUPBR_CHECK_CUDA(pt_launch_camera(F, W, st));
        CUPBR_CHECK_CUDA(mark());
        for (uint32_t d = 0; d < depth; ++d) {
            CUPBR_CHECK_CUDA(pt_launch_tail(s->g.dev, F, W, C, d, sms, st));
            if (d == 0) CUPBR_CHECK_CUDA(pt_launch_extend_camera(s->g.dev, W, sms, st, C.tail_threshold));
            else CUPBR_CHECK_CUDA(pt_launch_extend(s->g.dev, W, d, sms, st, C.tail_threshold));
            CUPBR_CHECK_CUDA(mark());
            CUPBR_CHECK_CUDA(pt_shade_cached(s->g.dev, F, W, C, d, sms, st));
            CUPBR_CHECK_CUDA(mark());
            CUPBR_CHECK_CUDA(pt_launch_connect(s->g.dev, W, d, sms, st));
            CUPBR_CHECK_CUDA(mark());
        }
        CUPBR_CHECK_CUDA(rc_infer_queries(c->net, c->infer_weights(), c->bounds, c->queries, c->counters, F.n_paths,
                                          W.radiance, sms, st));
        CUPBR_CHECK_CUDA(mark());
        CUPBR_CHECK_CUDA(pt_launch_accumulate(F, W, img, st));
        if (stride) CUPBR_CHECK_CUDA(rc_collect(F, W, C, c->samples, c->counters + 1, c->sample_capacity, st));
        CUPBR_CHECK_CUDA(mark());
        if (stride)
            for (uint32_t k = 0; k < steps; ++k)
                CUPBR_CHECK_CUDA(rc_train_step(c->net, c->bounds, c->samples, c->counters + 1, c->sample_capacity,
                                               k * c->desc.batch, steps * c->desc.batch, c->desc.batch, c->adam(),
                                               st));
        CUPBR_CHECK_CUDA(mark());
        if (c->profiling) c->ev_frames.push_back(std::move(ev));
    }
    return CUPBR_OK;
}
int cupbr_cache_get_counters(cupbr_cache_t c, uint32_t* out) {
    if (!c || !out) return fail(CUPBR_ERR_ARG, "null argument");
    CUPBR_CHECK_CUDA(cudaDeviceSynchronize());
    uint32_t err[2];
    CUPBR_CHECK_CUDA(cudaMemcpy(err, c->net.err, sizeof err, cudaMemcpyDeviceToHost));
    if (err[1]) c->lost = true;
    out[0] = err[0];
    CUPBR_CHECK_CUDA(cudaMemcpy(out + 1, c->counters, sizeof(uint32_t) * 2, cudaMemcpyDeviceToHost));
    return CUPBR_OK;
}
int cupbr_cache_check(cupbr_cache_t c, void* stream) {
    if (!c) return fail(CUPBR_ERR_ARG, "null cache");
    CUPBR_CHECK_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    uint32_t err[2];
    CUPBR_CHECK_CUDA(cudaMemcpy(err, c->net.err, sizeof err, cudaMemcpyDeviceToHost));
    if (err[1]) c->lost = true;
    if (c->lost) return fail(CUPBR_ERR_STATE, kCacheLost);
    if (err[0] == 0) return CUPBR_OK;
    CUPBR_CHECK_CUDA(cudaMemset(c->net.err, 0, sizeof(uint32_t)));
    return fail(CUPBR_ERR_TIMEOUT, "a tensor-core wait ran out of time (" + std::to_string(err[0]) +
                                       " CTAs gave up); the results of the calls since the last check are void");
}
int cupbr_cache_set_wait_probe(cupbr_cache_t c, uint32_t ns) {
    if (!c) return fail(CUPBR_ERR_ARG, "null cache");
    c->net.wait_probe_ns = ns;
    return CUPBR_OK;
}
int cupbr_cache_set_tail_paths(cupbr_cache_t c, uint32_t paths) {
    if (!c) return fail(CUPBR_ERR_ARG, "null cache");
    c->tail_paths = paths;
    return CUPBR_OK;
}
int cupbr_cache_set_batch_paths(cupbr_cache_t c, uint32_t paths) {
    if (!c || paths == 0) return fail(CUPBR_ERR_ARG, "batch must hold at least one path");
    c->batch_paths = paths;
    return CUPBR_OK;
}
int cupbr_cache_set_profiling(cupbr_cache_t c, int32_t enable) {
    if (!c) return fail(CUPBR_ERR_ARG, "null cache");
    c->profiling = enable != 0;
    // events created up front, outside the caller's timed region
    while (c->profiling && c->ev_pool.size() < 2048) {
        cudaEvent_t e;
        CUPBR_CHECK_CUDA(cudaEventCreate(&e));
        c->ev_pool.push_back(e);
    }
    return CUPBR_OK;
}
int cupbr_cache_get_stage_times(cupbr_cache_t c, float* ms7, uint32_t* waves) {
    if (!c || !ms7) return fail(CUPBR_ERR_ARG, "null argument");
    for (int k = 0; k < 7; ++k) ms7[k] = 0.0f;
    for (auto& e : c->ev_frames) {
        const size_t depth = (e.size() - 5) / 3;
        CUPBR_CHECK_CUDA(cudaEventSynchronize(e.back()));
        float t;
        CUPBR_CHECK_CUDA(cudaEventElapsedTime(&t, e[0], e[1]));
        ms7[0] += t;
        for (size_t d = 0; d < depth; ++d)
            for (int k = 0; k < 3; ++k) {
                CUPBR_CHECK_CUDA(cudaEventElapsedTime(&t, e[1 + 3 * d + k], e[2 + 3 * d + k]));
                ms7[1 + k] += t;
            }
        for (int k = 0; k < 3; ++k) {
            CUPBR_CHECK_CUDA(cudaEventElapsedTime(&t, e[1 + 3 * depth + k], e[2 + 3 * depth + k]));
            ms7[4 + k] += t;
        }
    }
    if (waves) *waves = (uint32_t)c->ev_frames.size();
    for (auto& e : c->ev_frames) c->ev_pool.insert(c->ev_pool.end(), e.begin(), e.end());
    c->ev_frames.clear();
    return CUPBR_OK;
}

int cupbr_device_alloc(void** p, size_t bytes) {
    if (!p) return fail(CUPBR_ERR_ARG, "null output");
    CUPBR_CHECK_CUDA(dev_alloc(p, bytes));
    return CUPBR_OK;
}
int cupbr_device_free(void* p) {
    CUPBR_CHECK_CUDA(cudaFree(p));
    return CUPBR_OK;
}
int cupbr_memcpy_h2d(void* dst, const void* src, size_t bytes, void* stream) {
    CUPBR_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream));
    return CUPBR_OK;
}
int cupbr_memcpy_d2h(void* dst, const void* src, size_t bytes, void* stream) {
    CUPBR_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    return CUPBR_OK;
}
int cupbr_stream_synchronize(void* stream) {
    CUPBR_CHECK_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return CUPBR_OK;
}
int cupbr_save_bmp(const char* path, const uint8_t* rgba, uint32_t w, uint32_t h) {
    std::string err;
    if (!path || !rgba) return fail(CUPBR_ERR_ARG, "null argument");
    return write_bmp_rgba(path, rgba, w, h, false, err) ? CUPBR_OK : fail(CUPBR_ERR_IO, err);
}
int cupbr_save_pfm(const char* path, const float* rgb, uint32_t w, uint32_t h) {
    std::string err;
    if (!path || !rgb) return fail(CUPBR_ERR_ARG, "null argument");
    return write_pfm(path, rgb, w, h, err) ? CUPBR_OK : fail(CUPBR_ERR_IO, err);
}

}  // extern "C"

// ------------------------------------------------ allocation failure hook ---
namespace cupbr_b200 {
namespace {
std::atomic<int64_t> g_alloc_fail_after{-1};
}  // namespace

cudaError_t dev_alloc(void** p, size_t bytes) {
    int64_t n = g_alloc_fail_after.load(std::memory_order_relaxed);
    while (n >= 0) {
        if (g_alloc_fail_after.compare_exchange_weak(n, n - 1)) {
            if (n == 0) {
                *p = nullptr;
                return cudaErrorMemoryAllocation;
            }
            break;
        }
    }
    return cudaMalloc(p, bytes);
}

void dev_alloc_fail_after(int64_t n) { g_alloc_fail_after.store(n < 0 ? -1 : n); }

}  // namespace cupbr_b200

extern "C" int cupbr_debug_fail_allocation(int64_t n) {
    cupbr_b200::dev_alloc_fail_after(n);
    return CUPBR_OK;
}
