/* cupbr-b200 C ABI: the drop-in boundary for cupbr's rendering hot path.
 *
 * Every entry point returns an int status (CUPBR_OK = 0; negative on error)
 * and records a message readable with cupbr_last_error().  No CUDA or C++
 * types cross this boundary: device buffers are plain pointers, streams are
 * `void*` (a cudaStream_t, NULL = the legacy default stream).
 *
 * Each declaration names the reference interface it replaces (paths are
 * relative to the cupbr project root).  Renderer, tone mapper and post
 * processor handles are not thread safe, like their reference counterparts
 * (single host thread, PBRenderer.cu / ToneMapper.cu / PostProcessor.cpp).
 */
#ifndef CUPBR_C_H
#define CUPBR_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUPBR_OK 0
#define CUPBR_ERR_ARG -1      /* bad argument / precondition (PBRenderer.cu:140-150 printed these) */
#define CUPBR_ERR_CUDA -2     /* CUDA runtime error */
#define CUPBR_ERR_IO -3       /* file parse / read / write error */
#define CUPBR_ERR_STATE -4    /* call not valid in the current state */
#define CUPBR_ERR_UNSUPPORTED -5 /* method disabled or not supported (PBRenderer.cu:161-191) */
#define CUPBR_ERR_TIMEOUT -6  /* a bounded wait inside a kernel ran out; that work's results are void */

/* enum class RenderingMethod, lib/include/Renderer/PBRenderer.h:14-22 */
enum cupbr_rendering_method {
    CUPBR_RAYTRACER = 0,
    CUPBR_WHITTED = 1,
    CUPBR_PATHTRACER = 2,
    CUPBR_METROPOLIS = 3,
    CUPBR_GRADIENTDOMAIN = 4,
    CUPBR_VOLUME = 5
};
/* enum class GeometryType, lib/include/Geometry/Geometry.h:15-23 */
enum cupbr_geometry_type { CUPBR_SPHERE = 0, CUPBR_PLANE = 1, CUPBR_QUAD = 2, CUPBR_TRIANGLE = 3, CUPBR_MESH = 4 };
/* enum class MaterialType, lib/include/Geometry/Material.h:14-22 */
enum cupbr_material_type {
    CUPBR_LAMBERT = 0, CUPBR_PHONG = 1, CUPBR_MIRROR = 2, CUPBR_GLASS = 3, CUPBR_GGX = 4, CUPBR_MAT_VOLUME = 5
};
/* enum LightType, lib/include/DataStructure/Light.h:11-15 */
enum cupbr_light_type { CUPBR_POINT = 0, CUPBR_AREA = 1 };
/* enum class ToneMappingType, lib/include/Renderer/ToneMapper.h:14-18 */
enum cupbr_tonemapping_type { CUPBR_REINHARD = 0, CUPBR_GAMMA = 1 };

typedef struct { float x, y, z; } cupbr_vec3;

/* class Material, lib/include/Geometry/Material.h:27-42 plus struct Volume,
 * lib/include/DataStructure/Volume.h:15-21.  cupbr_material_default() gives
 * the reference's member defaults. */
typedef struct {
    int32_t type;
    cupbr_vec3 albedo_e, albedo_d, albedo_s;
    float shininess, roughness, eta;
    cupbr_vec3 sigma_s, sigma_a;
    float g;
    int32_t interface_glass; /* Interface::GLASS */
} cupbr_material;

/* class Light, lib/include/DataStructure/Light.h:20-36 (half extents) */
typedef struct {
    int32_t type;
    cupbr_vec3 position, intensity, radiance, half_extend1, half_extend2;
} cupbr_light;

/* class Camera pose, lib/include/DataStructure/Camera.h:71-75 and
 * Camera::moved() (:59-60).  A moved camera restarts accumulation. */
typedef struct {
    cupbr_vec3 position, x_axis, y_axis, z_axis;
    float aspect_ratio;
    int32_t moved;
} cupbr_camera;

/* BVH build parameters (the reference's object BVH takes none). */
typedef struct {
    int32_t max_leaf_size;   /* primitives per leaf, 1..8 (default 4) */
    float traversal_cost;    /* SAH node-step cost relative to a primitive test (default 2) */
    int32_t top_bfs_levels;  /* 4-wide levels laid out breadth first for shared-memory staging, 0..8 (default 4) */
    int32_t builder;         /* CUPBR_BVH_BUILD_DEVICE (default): built on the GPU (level-parallel binning, one
                                CTA per small subtree); CUPBR_BVH_BUILD_HOST: on the host's threads.  Both give the
                                same node array and primitive order. */
} cupbr_bvh_params;
#define CUPBR_BVH_BUILD_DEVICE 0
#define CUPBR_BVH_BUILD_HOST 1

typedef struct {
    uint32_t objects, lights, triangles, spheres, quads, planes;
    uint32_t bvh_nodes, bvh_leaves, bvh_depth;
    double bvh_sah_cost;
    uint64_t device_bytes;
    uint32_t env_width, env_height;
    int32_t committed;
    int32_t bvh_builder;   /* CUPBR_BVH_BUILD_HOST or CUPBR_BVH_BUILD_DEVICE */
    double bvh_build_ms;   /* wall time of the BVH build in the last commit */
    double commit_ms;      /* wall time of the whole commit (boxes, BVH, tables, upload) */
} cupbr_scene_info;

/* one object as stored (for inspection / tests) */
typedef struct {
    int32_t type;
    cupbr_material material;
    cupbr_vec3 p0, p1, p2, p3; /* SPHERE center | PLANE pos,normal | QUAD pos,normal,extend1,extend2 */
    float radius;
    uint32_t triangle_begin, triangle_count;
    int32_t finite_box;
    cupbr_vec3 box_lo, box_hi;
} cupbr_object_desc;

typedef struct cupbr_scene_s* cupbr_scene_t;
typedef struct cupbr_renderer_s* cupbr_renderer_t;
typedef struct cupbr_tonemapper_s* cupbr_tonemapper_t;
typedef struct cupbr_postprocessor_s* cupbr_postprocessor_t;

/* ------------------------------------------------------------- errors --- */
/* Message of the last failing call on this thread (empty if none). */
const char* cupbr_last_error(void);
/* Library version string. */
const char* cupbr_version(void);

/* --------------------------------------------------------------- scene --- */
/* Material defaults, Material.h:34-42 / Volume.h:17-20. */
int cupbr_material_default(cupbr_material* out);
/* Camera(width, height), lib/src/DataStructure/Camera.cpp:6-11. */
int cupbr_camera_default(uint32_t width, uint32_t height, cupbr_camera* out);

/* SceneLoader::loadFromFile, lib/src/Scene/SceneLoader.cpp:140-454 (parse,
 * build and upload; the returned scene is committed). */
int cupbr_scene_load_xml(const char* path, cupbr_scene_t* out);
/* SceneLoader::loadFromFile with explicit BVH parameters (NULL = defaults). */
int cupbr_scene_load_xml_ex(const char* path, const cupbr_bvh_params* params, cupbr_scene_t* out);
/* The parsing half of SceneLoader::loadFromFile: objects, lights, volume and
 * environment are read (OBJ meshes and images included) but nothing is
 * built or uploaded; the scene stays editable until cupbr_scene_commit. */
int cupbr_scene_parse_xml(const char* path, cupbr_scene_t* out);
/* An empty scene to be filled by the add_* calls (the per-type branches of
 * SceneLoader.cpp:171-270) and then committed. */
int cupbr_scene_create(cupbr_scene_t* out);
/* new Sphere(position, radius), SceneLoader.cpp:199-210 / Sphere.h:25 */
int cupbr_scene_add_sphere(cupbr_scene_t s, cupbr_vec3 position, float radius, const cupbr_material* m, uint32_t* id);
/* new Plane(position, normal), SceneLoader.cpp:186-198 / Plane.h:24 */
int cupbr_scene_add_plane(cupbr_scene_t s, cupbr_vec3 position, cupbr_vec3 normal, const cupbr_material* m, uint32_t* id);
/* new Quad(position, normal, extend1, extend2), SceneLoader.cpp:211-228 / Quad.h:27 */
int cupbr_scene_add_quad(cupbr_scene_t s, cupbr_vec3 position, cupbr_vec3 normal, cupbr_vec3 extend1, cupbr_vec3 extend2,
                         const cupbr_material* m, uint32_t* id);
/* new Triangle(v1, v2, v3), SceneLoader.cpp:229-244 / Triangle.h:26 */
int cupbr_scene_add_triangle(cupbr_scene_t s, cupbr_vec3 v1, cupbr_vec3 v2, cupbr_vec3 v3, const cupbr_material* m,
                             uint32_t* id);
/* ObjLoader::loadObj result as arrays (lib/src/Scene/ObjLoader.cpp:13-87):
 * vertices (3 floats each) are transformed as scale * v + position; the
 * object's box spans all vertices. */
int cupbr_scene_add_mesh(cupbr_scene_t s, const float* vertices, uint32_t n_vertices, const uint32_t* indices,
                         uint32_t n_triangles, cupbr_vec3 position, cupbr_vec3 scale, const cupbr_material* m,
                         uint32_t* id);
/* ObjLoader::loadObj(path, position, scale), SceneLoader.cpp:245-262 */
int cupbr_scene_add_mesh_obj(cupbr_scene_t s, const char* path, cupbr_vec3 position, cupbr_vec3 scale,
                             const cupbr_material* m, uint32_t* id);
/* <lights><lightN>, SceneLoader.cpp:272-328 */
int cupbr_scene_add_light(cupbr_scene_t s, const cupbr_light* light);
/* <volume>, SceneLoader.cpp:330-344 (the default is sigma_s = sigma_a = 1, g = 0) */
int cupbr_scene_set_volume(cupbr_scene_t s, cupbr_vec3 sigma_s, cupbr_vec3 sigma_a, float g);
/* <environment>, SceneLoader.cpp:346-368: latitude-longitude RGB float image */
int cupbr_scene_set_environment(cupbr_scene_t s, const float* rgb, uint32_t width, uint32_t height);
/* Albedo texture of the scene (no counterpart in the reference, whose
 * materials have constant albedos): width*height RGB floats, row v, column
 * u, finite and >= 0.  Objects bound to it with cupbr_scene_set_object_texture
 * whose material is LAMBERT take their diffuse albedo from the texel their
 * planar projection puts the hit point on (nearest texel):
 *   u = dot(P - origin, u_axis) / |u_axis|^2, v = dot(P - origin, v_axis) / |v_axis|^2,
 * each clamped to [0, 1], texel (min(u * width, width - 1), min(v * height, height - 1)).
 * The path tracer (both estimators, pipelined or not, its tail kernel), the
 * radiance cache's renderer and the batch use it; VOLUME, GRADIENTDOMAIN,
 * RAYTRACER and the density-grid medium keep the materials' own albedos.
 * Before commit. */
int cupbr_scene_set_albedo_texture(cupbr_scene_t s, const float* rgb, uint32_t width, uint32_t height);
int cupbr_scene_set_object_texture(cupbr_scene_t s, uint32_t object, cupbr_vec3 origin, cupbr_vec3 u_axis,
                                   cupbr_vec3 v_axis);
/* The committed texture on the device: width*height texels of 4 floats
 * (RGB, one unused), row by row; NULL without a texture.  Writes to it
 * (on the device, ordered before the next render) change the albedos the
 * renderers use, e.g. a gradient step on the texture. */
int cupbr_scene_get_albedo_texture(cupbr_scene_t s, float** device_texels, uint32_t* width, uint32_t* height);
int cupbr_scene_load_environment(cupbr_scene_t s, const char* path); /* Radiance .hdr or .pfm */
/* Device upload + BVH build (SceneLoader.cpp:370-453). NULL params = defaults. */
int cupbr_scene_commit(cupbr_scene_t s, const cupbr_bvh_params* params);
/* SceneLoader::destroyScene, SceneLoader.cpp:456-522 */
int cupbr_scene_destroy(cupbr_scene_t s);
int cupbr_scene_get_info(cupbr_scene_t s, cupbr_scene_info* out);
int cupbr_scene_get_object(cupbr_scene_t s, uint32_t index, cupbr_object_desc* out);
int cupbr_scene_get_triangles(cupbr_scene_t s, uint32_t index, float* out_vertices, uint32_t capacity_triangles);
/* The committed scene's BVH as the traversal kernels read it: *n_nodes
 * 4-wide nodes of 32 floats each (x/y/z bounds of the four children, then
 * their references; bvh_build.hpp), copied to out_nodes when it is not NULL
 * and capacity_nodes >= *n_nodes.  Replaces the reference's host-side
 * object BVH (BoundingVolumeHierarchy.cpp:46-136) as the thing to inspect. */
int cupbr_scene_get_bvh(cupbr_scene_t s, float* out_nodes, uint32_t capacity_nodes, uint32_t* n_nodes);
/* Per primitive key (objects in the leaf order of the reference's object
 * BVH, BoundingVolumeHierarchy.cpp:46-136, then triangle index,
 * MeshDetail.h:28-35): the slot of its primitive in its type's table, i.e.
 * the BVH leaf order.
 * Copied to out when it is not NULL and capacity >= *n_keys. */
int cupbr_scene_get_key_slots(cupbr_scene_t s, uint32_t* out, uint32_t capacity, uint32_t* n_keys);
/* The scene file's <camera> element (an extension of the reference's XML:
 * <position>x,y,z</position> and either <yaw>/<pitch> in radians or
 * <look_at>x,y,z</look_at>) as the Camera a width x height view gets: axes
 * as Camera.cpp:82-88 builds them from yaw / pitch.  Without the element,
 * the default Camera(width, height) of Camera.cpp:6-11. */
int cupbr_scene_get_camera(cupbr_scene_t s, uint32_t width, uint32_t height, cupbr_camera* out);
/* Sets the scene's camera pose (the reference Camera's state: position, yaw, pitch). */
int cupbr_scene_set_camera(cupbr_scene_t s, cupbr_vec3 position, float yaw, float pitch);
int cupbr_scene_get_light(cupbr_scene_t s, uint32_t index, cupbr_light* out);
/* Tracing::traceRay (lib/src/Core/TracingDetail.h:47-66) for n host rays:
 * depth (INFINITY on miss), object id (scene_index, -1 on miss) and the
 * triangle index inside a MESH (-1 otherwise).  Directions are normalized
 * as the Ray constructor does (RayDetail.h:8-14). */
int cupbr_scene_trace(cupbr_scene_t s, uint32_t n, const float* origins, const float* directions, float* depth,
                      int32_t* object_id, int32_t* triangle_index);
/* Tracing::traceVisibility (TracingDetail.h:118-183) for n host rays. */
int cupbr_scene_visible(cupbr_scene_t s, uint32_t n, const float* origins, const float* directions,
                        const float* light_distance, int32_t* visible);
/* Interaction::pickMouse, lib/src/Interaction/MousePicker.cu:55-72: the
 * material and scene index of the object seen through pixel (x, y) of a
 * width x height view (un-jittered camera ray, TracingDetail.h:32-44).  On a
 * miss both outputs are left untouched, as in the reference. */
int cupbr_scene_pick(cupbr_scene_t s, const cupbr_camera* cam, uint32_t x, uint32_t y, uint32_t width,
                     uint32_t height, cupbr_material* out_material, int32_t* out_scene_index);
/* Interaction::updateMaterial, MousePicker.cu:74-81: replaces the material of
 * object scene_index (host copy and device copy) except its glass interface
 * flag, which the reference does not copy.  Renderers keep their
 * accumulated image; reset them to see the change alone. */
int cupbr_scene_update_material(cupbr_scene_t s, int32_t scene_index, const cupbr_material* m);

/* ------------------------------------------------------------ renderer --- */
/* PBRenderer(method), lib/include/Renderer/PBRenderer.h:36 */
int cupbr_renderer_create(int32_t method, cupbr_renderer_t* out);
/* PBRenderer::~PBRenderer */
int cupbr_renderer_destroy(cupbr_renderer_t r);
/* PBRenderer::setOutputSize, PBRenderer.cu:83-109 (buffers start zeroed) */
int cupbr_renderer_set_output_size(cupbr_renderer_t r, uint32_t width, uint32_t height);
/* PBRenderer::registerScene, PBRenderer.cu:111-116 (scene must be committed) */
int cupbr_renderer_register_scene(cupbr_renderer_t r, cupbr_scene_t s);
/* PBRenderer::setMethod, PBRenderer.cu:118-135: resets frameIndex, clears buffers */
int cupbr_renderer_set_method(cupbr_renderer_t r, int32_t method);
/* Estimator of PATHTRACER and VOLUME (no counterpart in the reference,
 * whose estimator is the default and the parity path).
 * CUPBR_ESTIMATOR_REFERENCE: pathtracer_kernel_nee / volume_kernel exactly
 *   (PathTracer.cu:20-95: the environment is counted twice, once through a
 *   BSDF-sampled "light" direction divided by its pdf and again when a path
 *   escapes; VolumeRenderer.cu:180-186: the scene medium's light term has no
 *   phase function).
 * CUPBR_ESTIMATOR_PHYSICAL: the environment's light term samples the
 *   environment map by its luminance and is weighted against BSDF sampling
 *   with the power heuristic, as is the radiance of an escaping path after a
 *   non-delta bounce (the same light pick as the reference; no environment
 *   light term at mirror, glass and volume-interface vertices); the scene
 *   medium's light term of VOLUME carries the Henyey-Greenstein phase value.
 *   Both estimators are unbiased for the scene's radiance here, the
 *   reference one is not where an environment is present.
 * Setting it restarts accumulation (frame index 0, image cleared). */
#define CUPBR_ESTIMATOR_REFERENCE 0
#define CUPBR_ESTIMATOR_PHYSICAL 1
int cupbr_renderer_set_estimator(cupbr_renderer_t r, int32_t estimator);
int cupbr_renderer_get_estimator(cupbr_renderer_t r, int32_t* estimator);
/* PBRenderer::getMethod */
int cupbr_renderer_get_method(cupbr_renderer_t r, int32_t* method);
/* PBRenderer::render(Camera*), PBRenderer.cu:137-230.  Enqueues one frame
 * (one sample per pixel folded into the running mean) on the renderer's
 * stream and returns without synchronizing. */
int cupbr_renderer_render(cupbr_renderer_t r, const cupbr_camera* camera);
/* nframes consecutive PBRenderer::render calls with the same camera (only
 * the first may restart accumulation when camera->moved).  The path tracer
 * and the VOLUME method render several frames per wavefront (up to the batch path budget, default
 * 33,554,432 paths: 16 frames of 1080p, 5.6 GB of wavefront state; long
 * queues at every depth keep the traversal kernels full) and folds them into
 * the running mean in frame order, so the image equals nframes single
 * render() calls.  The workspace grows to min(nframes, budget / pixels)
 * frames. */
int cupbr_renderer_render_frames(cupbr_renderer_t r, const cupbr_camera* camera, uint32_t nframes);
int cupbr_renderer_set_batch_paths(cupbr_renderer_t r, uint32_t paths);
/* PATHTRACER: once a depth's ray queue holds fewer than `paths` rays
 * (default 131,072 on one stream; off when pipelined, where the other
 * streams' frames fill the SMs a sparse queue leaves idle), one thread per
 * ray traces the rest of its path in one launch instead of a launch per
 * stage and depth (same image; 0 = off). */
int cupbr_renderer_set_tail_paths(cupbr_renderer_t r, uint32_t paths);
/* render_frames through one persistent-kernel launch instead of wavefronts
 * (no counterpart in the reference): each warp takes 32 pixels (an 8x4
 * tile) of the view and traces them through all n frames one thread per
 * path, the tile's camera rays as one warp packet, folding the frames into
 * the running mean in order -- the same image as the wavefronts, bit for
 * bit.  Used for PATHTRACER frames with the reference estimator and Russian
 * roulette off while profiling is off (otherwise the wavefronts run).  It
 * suits scenes that stay in L2, where the wavefront's queue traffic is the
 * larger cost; off by default. */
int cupbr_renderer_set_persistent(cupbr_renderer_t r, int32_t enable);
/* PATHTRACER, VOLUME and GRADIENTDOMAIN render(): with pipelining on, each
 * frame is traced on one of four internal streams (in turn) with its own
 * workspace and only its fold into the running mean (GRADIENTDOMAIN: the
 * means and the reconstruction) runs on the renderer's stream, in frame
 * order.  The
 * next render() calls can then trace while the caller still tone maps or
 * reads back earlier frames, and one frame's sparse last depths overlap the
 * next frames' first.  render_frames() alternates its (large) wavefronts
 * between the first two streams, so one wavefront's sparse last depths
 * overlap the next one's first (each still folded in frame order, after the
 * work queued on the renderer's stream when the call began).  Same images;
 * up to 4 extra wavefront workspaces.  Not used for profiled or instrumented
 * frames.  No counterpart in the reference (its render() is synchronous,
 * PBRenderer.cu:137-230). */
int cupbr_renderer_set_pipelined(cupbr_renderer_t r, int32_t enable);
/* PBRenderer::reset (frameIndex = 0) */
int cupbr_renderer_reset(cupbr_renderer_t r);
/* PBRenderer::setRussianRoulette (the reference leaves it uninitialised;
 * here the default is off) */
int cupbr_renderer_set_russian_roulette(cupbr_renderer_t r, int32_t enable);
/* PBRenderer::setMaxTraceDepth / getMaxTraceDepth (default 5, PBRenderer.cu:59) */
int cupbr_renderer_set_max_trace_depth(cupbr_renderer_t r, uint32_t depth);
int cupbr_renderer_get_max_trace_depth(cupbr_renderer_t r, uint32_t* depth);
/* PBRenderer::getOutputImage: device pointer to width*height RGB floats */
int cupbr_renderer_get_output(cupbr_renderer_t r, float** device_rgb, uint32_t* width, uint32_t* height);
/* PBRenderer::getGradientX / getGradientY (GRADIENTDOMAIN) */
int cupbr_renderer_get_gradient_x(cupbr_renderer_t r, float** device_rgb);
int cupbr_renderer_get_gradient_y(cupbr_renderer_t r, float** device_rgb);
/* The reconstruction half of PBRendering::gradientdomain
 * (GradientDomain.cu:382-401: init_kernel, then 50 optimization_kernel
 * passes each followed by the copy of temp into the output) on caller
 * buffers of width*height RGB floats: base and the four one-sided gradient
 * means in; gradient_x / gradient_y, temp and output written (temp's border
 * is read, never written, as in the reference: it lands in the output's). */
int cupbr_gdpt_reconstruct(uint32_t width, uint32_t height, const float* device_base, const float* device_gx_forward,
                           const float* device_gx_backward, const float* device_gy_forward,
                           const float* device_gy_backward, float* device_gradient_x, float* device_gradient_y,
                           float* device_temp, float* device_output, void* stream);
/* Progressive state for checkpoint / resume: the running mean is the output
 * image and the next frame index (PBRenderer.cu:35,46,184). */
int cupbr_renderer_get_frame_index(cupbr_renderer_t r, uint32_t* frame_index);
int cupbr_renderer_set_frame_index(cupbr_renderer_t r, uint32_t frame_index);
/* Stream all renderer work is enqueued on (cudaStream_t; NULL = legacy). */
int cupbr_renderer_set_stream(cupbr_renderer_t r, void* stream);
/* Counts of device-side errors seen so far (e.g. traversal stack overflow). */
int cupbr_renderer_get_error_count(cupbr_renderer_t r, uint32_t* count);
/* Traversal statistics: when enabled, frames count BVH node visits and
 * primitive tests (slower, for roofline accounting only).  stats[0..3] =
 * extension nodes, extension primitive tests, shadow nodes, shadow tests;
 * stats[4..5] = extension rays, shadow rays of the last frame. */
int cupbr_renderer_set_instrumented(cupbr_renderer_t r, int32_t enable);
int cupbr_renderer_get_stats(cupbr_renderer_t r, uint64_t* stats6);
/* Stage timing with CUDA events recorded on the renderer's stream around
 * every kernel of each frame rendered while profiling is on.
 * get_stage_times waits for those frames and returns the summed device
 * time of ms5 = {camera, extend (closest hit), shade, connect (shadow
 * rays), accumulate}, the frame count and the number of extend launches,
 * then forgets the frames.  Enabling creates a pool of 4,096 CUDA events up
 * front (a call outside any timed region), so profiled renders create none. */
int cupbr_renderer_set_profiling(cupbr_renderer_t r, int32_t enable);
int cupbr_renderer_get_stage_times(cupbr_renderer_t r, float* ms5, uint32_t* frames, uint32_t* extend_launches);

/* PBRendering::pathtracing, lib/include/Renderer/PathTracer.h:21-26: one
 * frame into a caller-owned device image (width*height RGB floats). */
int cupbr_pathtracing(cupbr_scene_t s, const cupbr_camera* camera, uint32_t frame_index, uint32_t max_trace_depth,
                      int32_t use_russian_roulette, float* device_rgb, uint32_t width, uint32_t height, void* stream);

/* ---------------------------------------------------------- tone map --- */
/* ToneMapper(type), lib/include/Renderer/ToneMapper.h:30 */
int cupbr_tonemapper_create(int32_t type, cupbr_tonemapper_t* out);
int cupbr_tonemapper_destroy(cupbr_tonemapper_t t);
/* ToneMapper::registerImage (ToneMapper.cu:118-130) */
int cupbr_tonemapper_register_image(cupbr_tonemapper_t t, const float* device_rgb, uint32_t width, uint32_t height);
/* ToneMapper::toneMap (ToneMapper.cu:132-165) */
int cupbr_tonemapper_tonemap(cupbr_tonemapper_t t);
/* ToneMapper::getRenderBuffer: device RGBA8 */
int cupbr_tonemapper_get_render_buffer(cupbr_tonemapper_t t, uint8_t** device_rgba, uint32_t* width, uint32_t* height);
int cupbr_tonemapper_get_type(cupbr_tonemapper_t t, int32_t* type);
int cupbr_tonemapper_set_type(cupbr_tonemapper_t t, int32_t type);
/* ToneMapper::setExposure (default 1, ToneMapper.cu:94) */
int cupbr_tonemapper_set_exposure(cupbr_tonemapper_t t, float exposure);
int cupbr_tonemapper_set_stream(cupbr_tonemapper_t t, void* stream);
/* ToneMapper::saveToFile (ToneMapper.cu:183-198): BMP, image row 0 at the bottom */
int cupbr_tonemapper_save_to_file(cupbr_tonemapper_t t, const char* path);
/* reinhard_kernel / gamma_kernel on caller buffers (ToneMapper.cu:17-69) */
int cupbr_tonemap(const float* device_rgb, uint32_t width, uint32_t height, int32_t type, float exposure,
                  uint8_t* device_rgba, void* stream);

/* Validation of the tone map's level tables (no counterpart in the
 * reference, which evaluates the formulas per pixel).  The tone map reads
 * each channel's 8-bit level from per-device tables built on the GPU from
 * the reference's formulas; the first tone-mapping call on a device enqueues
 * that build (about a millisecond) on its stream, and kernels that run before
 * it completes evaluate the formulas.  This call compares the looked-up level
 * with the formula's for every 32-bit float input: mismatches[t] = inputs
 * that differ (0 expected), flagged[t] = table buckets left to the formulas,
 * for t = REINHARD red/green, REINHARD blue, GAMMA.  Synchronizes the stream
 * (about 0.1 s). */
int cupbr_tonemap_verify_levels(uint64_t mismatches[3], uint32_t flagged[3], void* stream);

/* -------------------------------------------------------- post process --- */
/* PostProcessor, lib/include/PostProcessing/PostProcessor.h:12-52 */
int cupbr_postprocessor_create(cupbr_postprocessor_t* out);
int cupbr_postprocessor_destroy(cupbr_postprocessor_t p);
/* PostProcessor::registerImage (PostProcessor.cpp:108-118); width, height >= 2 */
int cupbr_postprocessor_register_image(cupbr_postprocessor_t p, const float* device_rgb, uint32_t width, uint32_t height);
/* PostProcessor::getPostProcessBuffer */
int cupbr_postprocessor_get_buffer(cupbr_postprocessor_t p, float** device_rgb);
/* PostProcessor::bloom(threshold), PostProcessor.cpp:125-142; threshold is
 * the curve (t, k - t, 2k, 0.25/k) of Interactor.cpp:436-440 */
int cupbr_postprocessor_bloom(cupbr_postprocessor_t p, const float threshold[4]);
int cupbr_postprocessor_set_stream(cupbr_postprocessor_t p, void* stream);
/* bloom followed by tone mapping in one pass over the output (no HDR write) */
int cupbr_postprocessor_bloom_tonemap(cupbr_postprocessor_t p, const float threshold[4], int32_t type, float exposure,
                                      uint8_t* device_rgba);

/* Bloom that allocates nothing.  No counterpart in the reference: it exists
 * for callers that cannot call cudaMalloc -- applications that reserve the
 * whole device memory budget up front and give it out themselves, and frame
 * loops that must not allocate after start-up because an allocation can
 * synchronize the device or fail mid-run.  Same result as
 * cupbr_postprocessor_bloom (PostProcessor::bloom semantics) on caller
 * buffers: device_rgb in, device_out out, width*height RGB floats each.
 * The half-resolution scratch is a fixed 12 MiB array inside the library,
 * held by every GPU that loads it until the process exits; the limit is
 * (width/2)*(height/2) <= 1048576 (inputs up to 2048x2048), larger images
 * are rejected with CUPBR_ERR_ARG.  The first call on a device looks up the
 * array's device address, so make that first call before any stream
 * capture.  All calls share the one array: calls whose GPU work overlaps
 * (two streams, two host threads) race and must be ordered by the caller.
 * The looked-up address is kept per device for the life of the process; a
 * cudaDeviceReset of a device invalidates it, so a process that resets a
 * device must not call this entry point on that device afterwards. */
int cupbr_bloom_noalloc(const float* device_rgb, uint32_t width, uint32_t height, const float threshold[4],
                        float* device_out, void* stream);

/* ------------------------------------------------- heterogeneous medium --- */
/* Density-grid medium rendered with delta / weighted tracking, and the
 * gradient of a loss on the image with respect to the densities and the
 * scene's albedos and light radiances by path replay.  No counterpart in the
 * reference: VolumeRenderer.cu renders a homogeneous medium only, and the
 * reference differentiates nothing.  Surfaces shade as in the path tracer
 * (PathTracer.cu:20-95); the medium fills the grid box (x fastest, then y,
 * then z; nearest-voxel lookup; zero density outside the box). */
typedef struct cupbr_medium_s* cupbr_medium_t;
typedef struct {
    uint32_t nx, ny, nz;      /* voxels */
    cupbr_vec3 lo, hi;        /* grid box in world space */
    float majorant;           /* >= every density of the grids passed in */
    float albedo;             /* scattering / extinction, in [0, 1] */
    float g;                  /* Henyey-Greenstein asymmetry, |g| < 1 */
    float q;                  /* 0: analog delta tracking (forward only);
                                 (0, 1): weighted tracking, real-event probability q */
} cupbr_medium_desc;

int cupbr_medium_create(const cupbr_medium_desc* desc, cupbr_medium_t* out);
int cupbr_medium_destroy(cupbr_medium_t m);
/* Length of the parameter gradient of a scene: 1 (medium albedo) + 3 per
 * object (diffuse albedo; Lambert objects, zero otherwise) + 3 per object
 * (emission albedo_e) + 3 per light (area light radiance or point light
 * intensity), in that order. */
int cupbr_medium_param_count(cupbr_scene_t s, uint32_t* out);
/* device_image (width*height RGB floats) = mean of spp samples, sample k of
 * pixel i seeded by tea(i, frame0 + k); device_density: nx*ny*nz floats. */
int cupbr_medium_forward(cupbr_medium_t m, cupbr_scene_t s, const float* device_density, const cupbr_camera* cam,
                         uint32_t width, uint32_t height, uint32_t spp, uint32_t frame0, uint32_t max_depth,
                         float* device_image, void* stream);
/* Adds dLoss/d(density) to device_grad_density (nx*ny*nz) and
 * dLoss/d(params) to device_grad_params (cupbr_medium_param_count floats)
 * for device_grad_image = dLoss/d(image) of the forward call with the same
 * arguments; the caller zeroes the gradients.  Needs 0 < q < 1. */
int cupbr_medium_backward(cupbr_medium_t m, cupbr_scene_t s, const float* device_density, const cupbr_camera* cam,
                          uint32_t width, uint32_t height, uint32_t spp, uint32_t frame0, uint32_t max_depth,
                          const float* device_grad_image, float* device_grad_density, float* device_grad_params,
                          void* stream);
/* Paths abandoned since creation (traversal stack overflow or a free flight
 * longer than 65536 steps); synchronizes the device. */
int cupbr_medium_get_error_count(cupbr_medium_t m, uint32_t* out);
/* Paths per wavefront (default 4,194,304; whole frames, at least one). */
int cupbr_medium_set_batch_paths(cupbr_medium_t m, uint32_t paths);
/* Forward calls made while profiling record CUDA events around every stage;
 * get_stage_times sums them (ms: camera, closest hit, shade, transmittance,
 * shadow rays, accumulation), gives the wavefront and shade-launch counts,
 * and clears. */
int cupbr_medium_set_profiling(cupbr_medium_t m, int32_t enable);
int cupbr_medium_get_stage_times(cupbr_medium_t m, float* ms6, uint32_t* wavefronts, uint32_t* shade_launches);
/* Forward calls made while instrumented count: [0] free-flight density
 * lookups, [1] ratio-tracking density lookups, [2] vertices shaded, [3]
 * shadow rays, [4] paths; get_stats reads and clears. */
int cupbr_medium_set_instrumented(cupbr_medium_t m, int32_t enable);
int cupbr_medium_get_stats(cupbr_medium_t m, uint64_t* stats5);

/* ------------------------------------------------------ batched views --- */
/* Many views (of one or more committed scenes, of any sizes and sample
 * counts) path traced by one launch captured as a CUDA graph and replayed
 * per launch.  No counterpart in the reference, where every view is its own
 * PBRenderer with one render() per frame (PBRenderer.cu:137-230): a launch
 * gives each view exactly what `spp` such render() calls give it -- frames
 * frame0 .. frame0 + spp - 1 folded into its running-mean image
 * (PathTracer.cu:162-168; frame0 = 0 starts a new mean), bit for bit.
 * Russian roulette off.  Scenes and images must outlive the batch and stay
 * committed.  Three modes (cupbr_batch_set_mode):
 * CUPBR_BATCH_PERSISTENT (default): the graph is one launch of a persistent
 *   kernel whose warps take work items -- 32 pixels (an 8x4 tile) of one
 *   view, of any scene, through all of that view's frames -- from one
 *   queue, heaviest first, and trace them one thread per path.
 * CUPBR_BATCH_WAVEFRONT: per scene, wavefronts of at most batch_paths paths
 *   through the path tracer's stage kernels (2 + 3 * max_depth launches each).
 * CUPBR_BATCH_COOPERATIVE: the wavefronts of CUPBR_BATCH_WAVEFRONT, every
 *   stage of every wavefront in one cooperative launch (256 threads per
 *   block, all blocks resident) with grid barriers between the stages.  A
 *   barrier that waits longer than 2 s ends the launch early (the views'
 *   images are then incomplete); cupbr_batch_get_error_count counts it
 *   until the next launch. */
#define CUPBR_BATCH_WAVEFRONT 0
#define CUPBR_BATCH_PERSISTENT 1
#define CUPBR_BATCH_COOPERATIVE 2
typedef struct {
    cupbr_scene_t scene;
    cupbr_camera camera;
    uint32_t width, height;
    uint32_t spp;          /* frames added per launch */
    uint32_t frame0;       /* frame index of the first of them */
    float* device_image;   /* width*height RGB running mean */
} cupbr_view;
typedef struct cupbr_batch_s* cupbr_batch_t;

int cupbr_batch_create(const cupbr_view* views, uint32_t n_views, uint32_t max_depth, cupbr_batch_t* out);
int cupbr_batch_destroy(cupbr_batch_t b);
/* Replays the graph on `stream` (uploads the view table first if frame0s changed). */
int cupbr_batch_launch(cupbr_batch_t b, void* stream);
/* frame0 += spp for every view: the next launch continues the means. */
int cupbr_batch_advance(cupbr_batch_t b);
int cupbr_batch_set_frame0(cupbr_batch_t b, uint32_t view, uint32_t frame0);
int cupbr_batch_get_info(cupbr_batch_t b, uint32_t* wavefronts, uint64_t* paths, uint32_t* kernel_launches,
                         uint32_t* batch_paths);
/* Wavefront and cooperative modes: paths per wavefront (default 4,194,304,
 * at least one frame of the largest view) and (wavefront mode) the share of
 * the traversal kernels' full occupancy (0, 1]; re-plans and re-captures
 * (the mode is unchanged). */
int cupbr_batch_configure(cupbr_batch_t b, uint32_t batch_paths, float trace_share);
/* Mode, and for the persistent kernel its block shape -- threads_per_block
 * 64, 128 or 256, blocks_per_sm resident blocks per SM (0: as many as fit;
 * larger values are clamped to that) -- and whether a warp finds the
 * closest hits of its 8x4 tile's camera rays as one packet (camera_packets
 * != 0, the default) or ray by ray (the same hits either way).  The
 * cooperative kernel takes threads_per_block 256 and blocks_per_sm as the
 * persistent kernel (camera rays always as packets).  Re-captures. */
int cupbr_batch_set_mode(cupbr_batch_t b, int32_t mode, uint32_t threads_per_block, uint32_t blocks_per_sm,
                         int32_t camera_packets);
int cupbr_batch_get_mode(cupbr_batch_t b, int32_t* mode, uint32_t* threads_per_block, uint32_t* blocks_per_sm,
                         int32_t* camera_packets);
/* Traversal stack overflows of the batch's launches and cooperative-mode
 * barrier timeouts (0 on a well-formed BVH). */
int cupbr_batch_get_error_count(cupbr_batch_t b, uint32_t* errors);
/* Test hook for the cooperative mode's bounded barrier waits: with ns > 0
 * (at most 1 s) one block of every launch leaves before the first grid
 * barrier, the others give up on it after ns nanoseconds and the launch ends
 * early with its timeout counted in cupbr_batch_get_error_count (no fault,
 * no hang).  0 (default) turns it off.  Re-captures in the cooperative mode. */
int cupbr_batch_set_barrier_probe(cupbr_batch_t b, uint64_t ns);
/* Autotuner: times every candidate as the median of three launches on
 * scratch images (the views' images are not touched) and keeps the fastest:
 * first the persistent kernel at 128 threads per block and full occupancy,
 * with and without camera packets, wavefronts of 2^21 .. 2^25 paths at
 * full traversal occupancy, and the cooperative kernel with wavefronts of
 * 2^22 and 2^24 paths; then around the best of those the persistent kernel
 * at 64 and 256 threads and at half occupancy, the best wavefront size at
 * 3/4 occupancy, or the cooperative kernel at half and twice its best
 * wavefront size.  With CUPBR_TUNE_BVH_LEAF the best configuration
 * is also timed with every scene's BVH rebuilt at leaf sizes 2 and 8 (the
 * scenes keep the fastest leaf size: images are the same for every BVH, but
 * every user of the scenes sees the rebuilt trees; other batches over them
 * notice the re-commit and rebuild their tables at their next launch).
 * Re-captures; synchronizes `stream`. */
#define CUPBR_TUNE_BVH_LEAF 1u
int cupbr_batch_autotune_ex(cupbr_batch_t b, void* stream, uint32_t flags, float* best_ms);
/* cupbr_batch_autotune_ex without flags. */
int cupbr_batch_autotune(cupbr_batch_t b, void* stream, float* best_ms);
/* Adjoint of a launch with respect to the scenes' albedo textures (no
 * counterpart in the reference, which differentiates nothing).
 * device_grad_images: one device pointer per view (width*height RGB floats
 * of dLoss/dImage, or 0 to skip the view).  Every path of the frames the
 * launch traced (frame0 .. frame0 + spp - 1 of each view) is re-traced from
 * its seed by the persistent kernel's work items; at each textured Lambert
 * vertex the derivative of the path's radiance with respect to that
 * vertex's texel -- (path radiance - radiance gathered before the vertex's
 * light term) / albedo per channel -- is scattered with weight
 * dLoss/dImage / (frame0 + spp), the weight of one frame in the running
 * mean.  The result is the gradient of sum(dLoss/dImage . image) with
 * respect to the texels for the frames of the launch (the whole image's
 * gradient when frame0 = 0).  Gradients are kept per scene by the batch
 * (cupbr_batch_get_texture_gradient): set with accumulate = 0, added to
 * otherwise.  max_depth <= 16.  Synchronizes `stream`. */
int cupbr_batch_backward(cupbr_batch_t b, const uint64_t* device_grad_images, int32_t accumulate, void* stream);
/* The gradient buffer of one of the batch's scenes: width*height RGB floats
 * (the scene's texture size), NULL before the first backward or for an
 * untextured scene. */
int cupbr_batch_get_texture_gradient(cupbr_batch_t b, cupbr_scene_t scene, float** device_grad_rgb, uint32_t* width,
                                     uint32_t* height);

/* ---------------------------------------------------- radiance cache --- */
/* Learned radiance cache.  No counterpart in the reference.  It is a
 * 96-64-64-64-64-64-3 ReLU MLP: 5 hidden layers of 64, FP16 weights and
 * activations, FP32 accumulation on the tensor cores.  It maps a path vertex
 * to the radiance leaving it towards the previous vertex.  Inputs:
 *   - position normalised to the scene box, sin/cos of pi 2^j x for
 *     12 bands per axis;
 *   - that direction, the shading normal, roughness and diffuse albedo;
 *   - a constant 1 and the bounces the path had left at the vertex.
 * A cached render path traces like PBRendering::pathtracing
 * (PathTracer.cu:97-169, Russian roulette off).  A path that is not a
 * training path ends at its first front-facing hit at depth >= cache_depth
 * that is not a mirror or glass (with cache_specular, beyond cache_depth: any
 * hit), and takes throughput * cache there instead of the
 * vertex's emission, direct light and continuation.  One path in
 * train_stride per frame is traced in full; its vertices give the training
 * samples, which train the cache online after each frame.
 *
 * Records are 5 float4 (80 bytes):
 *   [0] position, w: -
 *   [1] direction towards the previous vertex, w: roughness
 *   [2] normal, w: bounces left (max trace depth - vertex depth)
 *   [3] diffuse albedo, w: -
 *   [4] training samples: target RGB radiance, w: weight (0 or 1); inference: -
 * Parameters are layer-major, each layer row-major [out][in]:
 * 64x96, 4 x 64x64, then 3x64. */
typedef struct cupbr_cache_s* cupbr_cache_t;
typedef struct {
    uint32_t cache_depth;        /* first depth (0 = primary hit) the cache may answer */
    uint32_t train_stride;       /* one training path per train_stride paths (0: no online training) */
    uint32_t batch;              /* samples per Adam step, multiple of 128 (default 16384) */
    uint32_t samples_per_frame;  /* samples trained on per rendered frame, multiple of batch (default 65536) */
    float learning_rate;         /* Adam (default 1e-2, beta1 0.9, beta2 0.99, eps 1e-15) */
    uint32_t seed;               /* weight initialisation */
    uint32_t loss;               /* 0: relative L2 w (y - t)^2 / (y^2 + 0.01), y^2 held constant; 1: L2 */
    float weight_average;        /* decay of the weight average inference uses once training has
                                    stepped (0: the latest weights) */
    uint32_t cache_specular;     /* != 0: mirror and glass vertices deeper than cache_depth are answered too */
    uint32_t train_suffix;       /* 0: training paths are traced in full; k > 0: they end in a cache query
                                    at their first answerable hit at depth >= cache_depth + k */
} cupbr_cache_desc;

/* Sizes the position encoding to the committed scene's bounding box. */
int cupbr_cache_create(cupbr_scene_t scene, const cupbr_cache_desc* desc, cupbr_cache_t* out);
int cupbr_cache_destroy(cupbr_cache_t c);
uint32_t cupbr_cache_param_count(void);
/* The box positions are normalised to: x' = (x - lo) * inv_extent, clamped to [0, 1]. */
int cupbr_cache_get_bounds(cupbr_cache_t c, float* lo3, float* inv_extent3);
/* Host copies of the FP32 master weights; set also clears the Adam state. */
int cupbr_cache_get_params(cupbr_cache_t c, float* host_params);
int cupbr_cache_set_params(cupbr_cache_t c, const float* host_params);
/* Weights and Adam state to / from a file. */
int cupbr_cache_save(cupbr_cache_t c, const char* path);
int cupbr_cache_load(cupbr_cache_t c, const char* path);
/* device_out[i] = (network RGB of record i, 0) for n device records. */
int cupbr_cache_infer(cupbr_cache_t c, const float* device_records, uint32_t n, float* device_out, void* stream);
/* One Adam step on n device training records (n a multiple of 128, at most batch). */
int cupbr_cache_train_step(cupbr_cache_t c, const float* device_samples, uint32_t n, void* stream);
/* Mean loss gradient of the last step (parameter layout) and its relative
 * L2 loss.  These reads, get_params and get_counters synchronize the device. */
int cupbr_cache_get_gradient(cupbr_cache_t c, float* host_grad);
int cupbr_cache_get_loss(cupbr_cache_t c, float* loss, float* weighted_samples);
/* frames consecutive frames frame0 .. of the cached path tracer folded into
 * the width*height RGB running mean at device_image (frame0 = 0 starts it);
 * train != 0: online training (samples_per_frame per frame) after every
 * wavefront.  Frames are traced several per wavefront, up to batch_paths
 * paths (default 33,554,432, at least one frame). */
int cupbr_cache_render(cupbr_cache_t c, cupbr_scene_t s, const cupbr_camera* cam, uint32_t width, uint32_t height,
                       uint32_t frame0, uint32_t frames, uint32_t max_depth, int32_t train, float* device_image,
                       void* stream);
/* Counters: [0] CTAs whose tensor-core wait ran out of time since the last
 * cupbr_cache_check (results of the calls that saw one are void), [1]
 * queries, [2] training samples of the last frame. */
int cupbr_cache_get_counters(cupbr_cache_t c, uint32_t* counters3);
/* Error check of the tensor-core kernels (no reference counterpart; the
 * reference has no cache).  Synchronizes `stream`, then returns
 * CUPBR_ERR_TIMEOUT if a tensor-core wait of this cache ran out (every wait
 * is bounded at 2 s; a CTA that gives up stops issuing, waits once more,
 * bounded, for its MMAs in flight, frees its tensor memory and returns) and
 * clears that count; the cache stays usable.  If that second wait ran out as
 * well, the cache is lost: this and every later call on it return
 * CUPBR_ERR_STATE. */
int cupbr_cache_check(cupbr_cache_t c, void* stream);
/* Test hook for the bounded waits: with ns > 0, every inference CTA first
 * waits on a barrier that nothing arrives on, gives up after ns nanoseconds
 * with no tensor-core work issued, and counts itself as a wait that ran out
 * (cupbr_cache_check then reports CUPBR_ERR_TIMEOUT).  0 (default) turns it off. */
int cupbr_cache_set_wait_probe(cupbr_cache_t c, uint32_t ns);
/* Paths per cached wavefront (whole frames, at least one; default
 * 33,554,432).  Training steps follow each wavefront. */
int cupbr_cache_set_batch_paths(cupbr_cache_t c, uint32_t paths);
/* Once a depth's ray queue holds fewer than `paths` rays (default 65,536),
 * one thread per ray traces the rest of its path in a single launch instead
 * of a launch per stage and depth (same results); 0 never does. */
int cupbr_cache_set_tail_paths(cupbr_cache_t c, uint32_t paths);
/* Stage timing of cupbr_cache_render wavefronts while enabled: ms7 =
 * camera, closest hit (all depths), shading (all depths), shadow rays (all
 * depths), cache inference, accumulation + sample collection, training;
 * summed over the wavefronts traced since the last read. */
int cupbr_cache_set_profiling(cupbr_cache_t c, int32_t enable);
int cupbr_cache_get_stage_times(cupbr_cache_t c, float* ms7, uint32_t* wavefronts);

/* ------------------------------------------------------------ helpers --- */
/* Test hook for allocation failures (no counterpart in the reference, whose
 * allocations are unchecked in release builds, CUDA.h:18-22): every device
 * allocation of the library goes through one allocator; with n >= 0 the
 * n-th allocation from now (0: the next one) fails as cudaMalloc does when
 * memory runs out (nothing allocated, cudaErrorMemoryAllocation), after
 * which the hook is off again; n < 0 turns it off.  The call that hits it
 * returns CUPBR_ERR_CUDA and keeps or releases what it had allocated with
 * its object, as on a real failure. */
int cupbr_debug_fail_allocation(int64_t n);
int cupbr_device_alloc(void** device_ptr, size_t bytes);
int cupbr_device_free(void* device_ptr);
int cupbr_memcpy_h2d(void* device_dst, const void* host_src, size_t bytes, void* stream);
int cupbr_memcpy_d2h(void* host_dst, const void* device_src, size_t bytes, void* stream);
int cupbr_stream_synchronize(void* stream);
/* BMP / PFM writers for host buffers (row 0 = bottom of the picture). */
int cupbr_save_bmp(const char* path, const uint8_t* host_rgba, uint32_t width, uint32_t height);
int cupbr_save_pfm(const char* path, const float* host_rgb, uint32_t width, uint32_t height);

#ifdef __cplusplus
}
#endif

#endif /* CUPBR_C_H */
