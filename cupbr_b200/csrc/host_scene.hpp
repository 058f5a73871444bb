// Host-side scene model of cupbr-b200: the objects, materials, lights,
// environment and medium that cupbr's scene XML describes
// (lib/src/Scene/SceneLoader.cpp:140-454, lib/include/Scene/Scene.h:15-34),
// kept as flat arrays until commit() builds the BVH and uploads them.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace cupbr_b200 {

// lib/include/Geometry/Geometry.h:15-23 (BVH omitted: it is not a scene object)
enum GeoType : int { GEO_SPHERE = 0, GEO_PLANE = 1, GEO_QUAD = 2, GEO_TRIANGLE = 3, GEO_MESH = 4 };
// lib/include/Geometry/Material.h:14-22
enum MatType : int { MAT_LAMBERT = 0, MAT_PHONG = 1, MAT_MIRROR = 2, MAT_GLASS = 3, MAT_GGX = 4, MAT_VOLUME = 5 };

// Field defaults follow Material.h:34-40 and Volume.h:15-21.
struct HMaterial {
    int type = MAT_LAMBERT;
    float albedo_e[3] = {0, 0, 0};
    float albedo_d[3] = {1, 1, 1};
    float albedo_s[3] = {0, 0, 0};
    float shininess = 128.0f * 0.4f;
    float roughness = 1.0f;
    float eta = 1.5f;
    float sigma_s[3] = {1, 1, 1};
    float sigma_a[3] = {1, 1, 1};
    float g = 0.0f;
    int interface_glass = 0;
};

struct HObject {
    int type = GEO_MESH;
    HMaterial mat;
    float p0[3] = {0, 0, 0}, p1[3] = {0, 0, 0}, p2[3] = {0, 0, 0}, p3[3] = {0, 0, 0};
    float radius = 0.0f;
    uint32_t tri_begin = 0, tri_count = 0;  // range in HostScene::tri_verts (9 floats each)
    // The reference's per-object box (Geometry.cu:6-10 infinite by default;
    // SphereDetail.h:16 and MeshDetail.h:18 set finite ones).
    bool finite_box = false;
    float box_lo[3] = {0, 0, 0}, box_hi[3] = {0, 0, 0};
    // Albedo texture binding (no counterpart in the reference): a textured
    // Lambert object takes its diffuse albedo from the scene's texture at
    // the planar projection u = dot(P - tex_origin, tex_u) / |tex_u|^2,
    // v = dot(P - tex_origin, tex_v) / |tex_v|^2 (clamped to [0, 1]).
    bool textured = false;
    float tex_origin[3] = {0, 0, 0}, tex_u[3] = {1, 0, 0}, tex_v[3] = {0, 0, 1};
};

// lib/include/DataStructure/Light.h:11-36
struct HLight {
    int type = 0;  // 0 POINT, 1 AREA
    float position[3] = {0, 0, 0}, intensity[3] = {0, 0, 0}, radiance[3] = {0, 0, 0};
    float he1[3] = {0, 0, 0}, he2[3] = {0, 0, 0};
};

// Camera pose of a scene file's optional <camera> element (an extension of
// the reference's schema): the reference Camera's own state, position plus
// yaw / pitch in radians (Camera.cpp:52-88; yaw pi/2, pitch 0 look along +z).
struct HCamera {
    bool set = false;
    float position[3] = {0, 0, 0};
    float yaw = 1.57079632679f, pitch = 0.0f;
};

struct HostScene {
    std::vector<HObject> objects;
    HCamera camera;
    std::vector<float> tri_verts;  // 9 floats per triangle (world space, after the mesh transform)
    std::vector<HLight> lights;
    std::vector<float> env;        // RGB float, env_w * env_h * 3
    uint32_t env_w = 0, env_h = 0;
    std::vector<float> tex;        // albedo texture, RGB float, tex_w * tex_h * 3 (row v, column u)
    uint32_t tex_w = 0, tex_h = 0;
    float vol_sigma_s[3] = {1, 1, 1}, vol_sigma_a[3] = {1, 1, 1}, vol_g = 0.0f;  // Scene.h:23 default Volume

    uint32_t add_sphere(const float pos[3], float radius, const HMaterial& m);
    uint32_t add_plane(const float pos[3], const float normal[3], const HMaterial& m);
    uint32_t add_quad(const float pos[3], const float normal[3], const float e1[3], const float e2[3], const HMaterial& m);
    uint32_t add_triangle(const float v1[3], const float v2[3], const float v3[3], const HMaterial& m);
    // ObjLoader.cpp:13-87 semantics: vertex' = scale * v + position, the box
    // spans ALL listed vertices.
    uint32_t add_mesh(const float* verts, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float pos[3],
                      const float scale[3], const HMaterial& m);
};

// XML / OBJ / image readers (scene_io.cpp).  Each returns false and fills err
// on malformed input instead of printing and continuing as the reference does.
bool load_scene_xml(const std::string& path, HostScene& out, std::string& err);
bool load_obj(const std::string& path, std::vector<float>& verts, std::vector<uint32_t>& idx, std::string& err);
bool load_hdr_image(const std::string& path, std::vector<float>& rgb, uint32_t& w, uint32_t& h, std::string& err);
bool write_bmp_rgba(const std::string& path, const uint8_t* rgba, uint32_t w, uint32_t h, bool flip, std::string& err);
bool write_pfm(const std::string& path, const float* rgb, uint32_t w, uint32_t h, std::string& err);
bool read_pfm(const std::string& path, std::vector<float>& rgb, uint32_t& w, uint32_t& h, std::string& err);

}  // namespace cupbr_b200
