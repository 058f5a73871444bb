// Scene XML, OBJ and image I/O for cupbr-b200 (host side).
//
// The XML schema is cupbr's (SceneLoader.cpp:140-454): several top-level
// elements <header>, <geometry>, <lights>, <volume>, <environment>; geometry
// and light entries are named geometry1..N / light1..N; vectors are written
// "x,y,z".  The reference parses with tinyxml2 (absent from its tree); this
// is a small reader of our own for that element-and-text subset.
#include "host_scene.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace cupbr_b200 {

namespace {

struct XNode {
    std::string name;
    std::string text;
    std::vector<XNode> children;
    const XNode* child(const char* n) const {
        for (const XNode& c : children)
            if (c.name == n) return &c;
        return nullptr;
    }
};

std::string trim(const std::string& s) {
    size_t b = s.find_first_not_of(" \t\r\n");
    if (b == std::string::npos) return "";
    size_t e = s.find_last_not_of(" \t\r\n");
    return s.substr(b, e - b + 1);
}

// Parses a sequence of elements (no DTD, no CDATA); comments and processing
// instructions are skipped; attributes are ignored.
class XmlReader {
  public:
    explicit XmlReader(const std::string& s) : s_(s) {}
    bool parse_all(XNode& root, std::string& err) {
        root.name = "#document";
        if (!parse_children(root, "", err)) return false;
        return true;
    }

  private:
    const std::string& s_;
    size_t i_ = 0;

    bool skip_misc() {
        for (;;) {
            if (s_.compare(i_, 4, "<!--") == 0) {
                size_t e = s_.find("-->", i_ + 4);
                if (e == std::string::npos) return false;
                i_ = e + 3;
            } else if (s_.compare(i_, 2, "<?") == 0) {
                size_t e = s_.find("?>", i_ + 2);
                if (e == std::string::npos) return false;
                i_ = e + 2;
            } else if (s_.compare(i_, 2, "<!") == 0) {
                size_t e = s_.find('>', i_ + 2);
                if (e == std::string::npos) return false;
                i_ = e + 1;
            } else {
                return true;
            }
        }
    }

    bool parse_children(XNode& parent, const std::string& close, std::string& err) {
        std::string text;
        while (i_ < s_.size()) {
            size_t lt = s_.find('<', i_);
            if (lt == std::string::npos) {
                text += s_.substr(i_);
                i_ = s_.size();
                break;
            }
            text += s_.substr(i_, lt - i_);
            i_ = lt;
            if (!skip_misc()) { err = "unterminated comment or declaration"; return false; }
            if (i_ >= s_.size() || s_[i_] != '<') continue;
            if (s_.compare(i_, 2, "</") == 0) {
                size_t e = s_.find('>', i_);
                if (e == std::string::npos) { err = "unterminated closing tag"; return false; }
                std::string nm = trim(s_.substr(i_ + 2, e - i_ - 2));
                if (nm != close) { err = "mismatched closing tag </" + nm + "> (expected </" + close + ">)"; return false; }
                i_ = e + 1;
                parent.text = trim(text);
                return true;
            }
            size_t e = s_.find('>', i_);
            if (e == std::string::npos) { err = "unterminated tag"; return false; }
            std::string inner = s_.substr(i_ + 1, e - i_ - 1);
            bool self_close = !inner.empty() && inner.back() == '/';
            if (self_close) inner.pop_back();
            inner = trim(inner);
            size_t sp = inner.find_first_of(" \t\r\n");
            XNode node;
            node.name = sp == std::string::npos ? inner : inner.substr(0, sp);
            if (node.name.empty()) { err = "empty tag name"; return false; }
            i_ = e + 1;
            if (!self_close && !parse_children(node, node.name, err)) return false;
            parent.children.push_back(std::move(node));
        }
        if (!close.empty()) { err = "missing closing tag </" + close + ">"; return false; }
        parent.text = trim(text);
        return true;
    }
};

// SceneLoader.cpp:21-33: comma separated floats through std::stof
bool vec3_of(const XNode* n, float out[3], std::string& err, const char* what) {
    if (!n) { err = std::string("missing <") + what + ">"; return false; }
    std::stringstream ss(n->text);
    std::string item;
    std::vector<float> r;
    while (std::getline(ss, item, ',')) {
        const char* b = item.c_str();
        char* e = nullptr;
        float v = std::strtof(b, &e);
        if (e == b) { err = std::string("bad number in <") + what + ">: '" + n->text + "'"; return false; }
        r.push_back(v);
    }
    if (r.size() < 3) { err = std::string("<") + what + "> needs three components: '" + n->text + "'"; return false; }
    out[0] = r[0]; out[1] = r[1]; out[2] = r[2];
    return true;
}

bool float_of(const XNode* n, float& out, std::string& err, const char* what) {
    if (!n) { err = std::string("missing <") + what + ">"; return false; }
    const char* b = n->text.c_str();
    char* e = nullptr;
    out = std::strtof(b, &e);
    if (e == b) { err = std::string("bad number in <") + what + ">"; return false; }
    return true;
}

bool uint_of(const XNode* n, uint32_t& out, std::string& err, const char* what) {
    if (!n) { err = std::string("missing <") + what + ">"; return false; }
    const char* b = n->text.c_str();
    char* e = nullptr;
    long v = std::strtol(b, &e, 10);
    if (e == b || v < 0) { err = std::string("bad count in <") + what + ">"; return false; }
    out = (uint32_t)v;
    return true;
}

// SceneLoader.cpp:35-137
bool material_of(const XNode* m, HMaterial& mat, std::string& err) {
    if (!m) { err = "missing <material>"; return false; }
    const XNode* t = m->child("type");
    if (!t) { err = "material without <type>"; return false; }
    static const char* names[] = {"LAMBERT", "PHONG", "MIRROR", "GLASS", "GGX", "VOLUME"};
    int type = -1;
    for (int i = 0; i < 6; ++i)
        if (t->text == names[i]) type = i;
    if (type < 0) { err = t->text + " is not a valid material type"; return false; }
    mat.type = type;
    if (const XNode* n = m->child("albedo_e")) { if (!vec3_of(n, mat.albedo_e, err, "albedo_e")) return false; }
    if (const XNode* n = m->child("albedo_d")) { if (!vec3_of(n, mat.albedo_d, err, "albedo_d")) return false; }
    if (const XNode* n = m->child("albedo_s")) { if (!vec3_of(n, mat.albedo_s, err, "albedo_s")) return false; }
    if (const XNode* n = m->child("shininess")) { if (!float_of(n, mat.shininess, err, "shininess")) return false; }
    if (const XNode* n = m->child("roughness")) {
        float r;
        if (!float_of(n, r, err, "roughness")) return false;
        mat.roughness = std::max(1e-4f, r);  // SceneLoader.cpp:104-107
    }
    if (const XNode* n = m->child("eta")) { if (!float_of(n, mat.eta, err, "eta")) return false; }
    if (const XNode* n = m->child("sigma_s")) { if (!vec3_of(n, mat.sigma_s, err, "sigma_s")) return false; }
    if (const XNode* n = m->child("sigma_a")) { if (!vec3_of(n, mat.sigma_a, err, "sigma_a")) return false; }
    if (const XNode* n = m->child("g")) { if (!float_of(n, mat.g, err, "g")) return false; }
    if (const XNode* n = m->child("interface")) mat.interface_glass = n->text == "GLASS" ? 1 : 0;
    return true;
}

std::string dir_of(const std::string& p) {
    size_t s = p.find_last_of('/');
    return s == std::string::npos ? std::string(".") : p.substr(0, s);
}

bool file_exists(const std::string& p) {
    FILE* f = std::fopen(p.c_str(), "rb");
    if (!f) return false;
    std::fclose(f);
    return true;
}

// The reference opens asset paths relative to the working directory
// (e.g. "res/Meshes/box.obj").  Try that first, then relative to the XML's
// directory and its ancestors.
std::string resolve(const std::string& asset, const std::string& xml_path) {
    if (asset.empty() || asset[0] == '/' || file_exists(asset)) return asset;
    std::string d = dir_of(xml_path);
    for (int up = 0; up < 4; ++up) {
        std::string cand = d + "/" + asset;
        if (file_exists(cand)) return cand;
        d += "/..";
    }
    return asset;
}

}  // namespace

bool load_scene_xml(const std::string& path, HostScene& sc, std::string& err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "failed to open scene file: " + path; return false; }
    std::stringstream buf;
    buf << f.rdbuf();
    std::string text = buf.str();
    XNode root;
    XmlReader rd(text);
    if (!rd.parse_all(root, err)) { err = path + ": " + err; return false; }

    const XNode* header = root.child("header");
    if (!header) { err = path + ": missing <header>"; return false; }
    uint32_t scene_size = 0, light_count = 0;
    if (!uint_of(header->child("scene_size"), scene_size, err, "scene_size")) return false;
    if (!uint_of(header->child("light_count"), light_count, err, "light_count")) return false;

    const XNode* geo = root.child("geometry");
    if (scene_size > 0 && !geo) { err = path + ": missing <geometry>"; return false; }
    for (uint32_t i = 0; i < scene_size; ++i) {
        std::string nm = "geometry" + std::to_string(i + 1);
        const XNode* g = geo->child(nm.c_str());
        if (!g) { err = path + ": missing <" + nm + ">"; return false; }
        const XNode* t = g->child("type");
        if (!t) { err = path + ": <" + nm + "> without <type>"; return false; }
        HMaterial mat;
        if (!material_of(g->child("material"), mat, err)) { err = path + ": <" + nm + ">: " + err; return false; }
        float a[3], b[3], c[3], d[3];
        if (t->text == "PLANE") {
            if (!vec3_of(g->child("position"), a, err, "position") || !vec3_of(g->child("normal"), b, err, "normal")) return false;
            sc.add_plane(a, b, mat);
        } else if (t->text == "SPHERE") {
            float r;
            if (!vec3_of(g->child("position"), a, err, "position") || !float_of(g->child("radius"), r, err, "radius")) return false;
            sc.add_sphere(a, r, mat);
        } else if (t->text == "QUAD") {
            if (!vec3_of(g->child("position"), a, err, "position") || !vec3_of(g->child("normal"), b, err, "normal") ||
                !vec3_of(g->child("extend1"), c, err, "extend1") || !vec3_of(g->child("extend2"), d, err, "extend2"))
                return false;
            sc.add_quad(a, b, c, d, mat);
        } else if (t->text == "TRIANGLE") {
            if (!vec3_of(g->child("vertex1"), a, err, "vertex1") || !vec3_of(g->child("vertex2"), b, err, "vertex2") ||
                !vec3_of(g->child("vertex3"), c, err, "vertex3"))
                return false;
            sc.add_triangle(a, b, c, mat);
        } else if (t->text == "MESH") {
            const XNode* p = g->child("path");
            if (!p) { err = path + ": <" + nm + "> MESH without <path>"; return false; }
            float pos[3] = {0, 0, 0}, scale[3] = {1, 1, 1};
            if (const XNode* n = g->child("position")) { if (!vec3_of(n, pos, err, "position")) return false; }
            if (const XNode* n = g->child("scale")) { if (!vec3_of(n, scale, err, "scale")) return false; }
            std::vector<float> v;
            std::vector<uint32_t> idx;
            if (!load_obj(resolve(p->text, path), v, idx, err)) return false;
            sc.add_mesh(v.data(), (uint32_t)(v.size() / 3), idx.data(), (uint32_t)(idx.size() / 3), pos, scale, mat);
        } else {
            err = path + ": " + t->text + " is not a valid geometry type";
            return false;
        }
    }

    const XNode* lh = root.child("lights");
    if (light_count > 0 && !lh) { err = path + ": missing <lights>"; return false; }
    for (uint32_t i = 0; i < light_count; ++i) {  // SceneLoader.cpp:272-328
        std::string nm = "light" + std::to_string(i + 1);
        const XNode* l = lh->child(nm.c_str());
        if (!l) { err = path + ": missing <" + nm + ">"; return false; }
        const XNode* t = l->child("type");
        HLight li;
        if (!t) { err = path + ": <" + nm + "> without <type>"; return false; }
        if (t->text == "POINT") li.type = 0;
        else if (t->text == "AREA") li.type = 1;
        else { err = path + ": " + t->text + " is not a valid light type"; return false; }
        if (const XNode* n = l->child("position")) { if (!vec3_of(n, li.position, err, "position")) return false; }
        if (const XNode* n = l->child("intensity")) { if (!vec3_of(n, li.intensity, err, "intensity")) return false; }
        if (const XNode* n = l->child("radiance")) { if (!vec3_of(n, li.radiance, err, "radiance")) return false; }
        if (const XNode* n = l->child("extend1")) { if (!vec3_of(n, li.he1, err, "extend1")) return false; }
        if (const XNode* n = l->child("extend2")) { if (!vec3_of(n, li.he2, err, "extend2")) return false; }
        sc.lights.push_back(li);
    }

    if (const XNode* c = root.child("camera")) {  // extension: <position>, then <yaw>/<pitch> or <look_at>
        HCamera& cam = sc.camera;
        cam.set = true;
        if (const XNode* n = c->child("position")) { if (!vec3_of(n, cam.position, err, "camera position")) return false; }
        const XNode* la = c->child("look_at");
        if (la) {
            float t[3];
            if (!vec3_of(la, t, err, "look_at")) return false;
            const double f[3] = {(double)t[0] - cam.position[0], (double)t[1] - cam.position[1],
                                 (double)t[2] - cam.position[2]};
            const double len = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
            if (!(len > 0.0)) { err = path + ": <camera> look_at equals its position"; return false; }
            // front = (cos yaw cos pitch, sin pitch, sin yaw cos pitch), Camera.cpp:82-84
            cam.pitch = (float)std::asin(std::max(-1.0, std::min(1.0, f[1] / len)));
            cam.yaw = (float)std::atan2(f[2], f[0]);
        }
        if (const XNode* n = c->child("yaw")) {
            if (la) { err = path + ": <camera> takes either <look_at> or <yaw>/<pitch>"; return false; }
            if (!float_of(n, cam.yaw, err, "yaw")) return false;
        }
        if (const XNode* n = c->child("pitch")) {
            if (la) { err = path + ": <camera> takes either <look_at> or <yaw>/<pitch>"; return false; }
            if (!float_of(n, cam.pitch, err, "pitch")) return false;
        }
        const float lim = 3.14159f / 2.0f;  // Camera.cpp:77-80
        cam.pitch = std::max(-lim, std::min(lim, cam.pitch));
    }

    if (const XNode* v = root.child("volume")) {  // SceneLoader.cpp:330-344
        if (!vec3_of(v->child("sigma_s"), sc.vol_sigma_s, err, "sigma_s") ||
            !vec3_of(v->child("sigma_a"), sc.vol_sigma_a, err, "sigma_a") || !float_of(v->child("g"), sc.vol_g, err, "g"))
            return false;
    }

    if (const XNode* e = root.child("environment")) {  // SceneLoader.cpp:346-368
        const XNode* p = e->child("path");
        if (!p) { err = path + ": <environment> without <path>"; return false; }
        std::string ep = resolve(p->text, path);
        bool ok;
        size_t n = ep.size();
        if (n > 4 && ep.compare(n - 4, 4, ".pfm") == 0) ok = read_pfm(ep, sc.env, sc.env_w, sc.env_h, err);
        else ok = load_hdr_image(ep, sc.env, sc.env_w, sc.env_h, err);
        if (!ok) return false;
    }
    return true;
}

// ObjLoader.cpp:13-87: "v x y z" and "f a/b/c a/b/c a/b/c" (first three
// vertex references of a face; the index before the first '/').
bool load_obj(const std::string& path, std::vector<float>& verts, std::vector<uint32_t>& idx, std::string& err) {
    std::ifstream f(path);
    if (!f) { err = "failed to open OBJ file: " + path; return false; }
    std::string line;
    size_t lineno = 0;
    while (std::getline(f, line)) {
        ++lineno;
        if (line.size() < 2) continue;
        if (line[0] == 'v' && line[1] == ' ') {
            const char* p = line.c_str() + 2;
            for (int k = 0; k < 3; ++k) {
                char* e = nullptr;
                float v = std::strtof(p, &e);
                if (e == p) { err = path + ":" + std::to_string(lineno) + ": bad vertex"; return false; }
                verts.push_back(v);
                p = e;
            }
        } else if (line[0] == 'f' && line[1] == ' ') {
            std::stringstream ss(line.substr(2));
            std::string tok;
            uint32_t got = 0, tri[3];
            while (got < 3 && ss >> tok) {
                long v = std::strtol(tok.c_str(), nullptr, 10);
                if (v <= 0) { err = path + ":" + std::to_string(lineno) + ": unsupported face index '" + tok + "'"; return false; }
                tri[got++] = (uint32_t)(v - 1);
            }
            if (got < 3) { err = path + ":" + std::to_string(lineno) + ": face with fewer than 3 vertices"; return false; }
            idx.insert(idx.end(), tri, tri + 3);
        }
    }
    uint32_t nv = (uint32_t)(verts.size() / 3);
    for (uint32_t i : idx)
        if (i >= nv) { err = path + ": face index out of range"; return false; }
    return true;
}

// Radiance RGBE (.hdr) reader: the format stbi_loadf decodes for the
// reference's environment maps (SceneLoader.cpp:352).  Flat and new-style
// run-length scanlines; "-Y h +X w" orientation.
bool load_hdr_image(const std::string& path, std::vector<float>& rgb, uint32_t& w, uint32_t& h, std::string& err) {
    FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) { err = "failed to open environment map: " + path; return false; }
    char line[512];
    if (!std::fgets(line, sizeof line, fp) || std::strncmp(line, "#?", 2) != 0) {
        std::fclose(fp);
        err = path + ": not a Radiance HDR file";
        return false;
    }
    while (std::fgets(line, sizeof line, fp))
        if (line[0] == '\n' || (line[0] == '\r' && line[1] == '\n')) break;
    int H = 0, W = 0;
    if (!std::fgets(line, sizeof line, fp) || std::sscanf(line, "-Y %d +X %d", &H, &W) != 2 || H <= 0 || W <= 0) {
        std::fclose(fp);
        err = path + ": unsupported HDR resolution line";
        return false;
    }
    w = (uint32_t)W;
    h = (uint32_t)H;
    rgb.assign((size_t)W * H * 3, 0.0f);
    std::vector<uint8_t> scan((size_t)W * 4);
    for (int y = 0; y < H; ++y) {
        int c0 = std::fgetc(fp), c1 = std::fgetc(fp), c2 = std::fgetc(fp), c3 = std::fgetc(fp);
        if (c3 == EOF) { std::fclose(fp); err = path + ": truncated"; return false; }
        if (c0 == 2 && c1 == 2 && ((c2 << 8) | c3) == W && W >= 8 && W < 32768) {
            for (int ch = 0; ch < 4; ++ch) {
                int x = 0;
                while (x < W) {
                    int cnt = std::fgetc(fp);
                    if (cnt == EOF) { std::fclose(fp); err = path + ": truncated"; return false; }
                    if (cnt > 128) {
                        cnt -= 128;
                        int val = std::fgetc(fp);
                        if (x + cnt > W) { std::fclose(fp); err = path + ": bad run"; return false; }
                        for (int k = 0; k < cnt; ++k) scan[(size_t)(x++) * 4 + ch] = (uint8_t)val;
                    } else {
                        if (cnt == 0 || x + cnt > W) { std::fclose(fp); err = path + ": bad run"; return false; }
                        for (int k = 0; k < cnt; ++k) scan[(size_t)(x++) * 4 + ch] = (uint8_t)std::fgetc(fp);
                    }
                }
            }
        } else {
            scan[0] = (uint8_t)c0; scan[1] = (uint8_t)c1; scan[2] = (uint8_t)c2; scan[3] = (uint8_t)c3;
            if (W > 1 && std::fread(scan.data() + 4, 1, (size_t)(W - 1) * 4, fp) != (size_t)(W - 1) * 4) {
                std::fclose(fp);
                err = path + ": truncated";
                return false;
            }
        }
        for (int x = 0; x < W; ++x) {
            const uint8_t* p = &scan[(size_t)x * 4];
            float* o = &rgb[((size_t)y * W + x) * 3];
            if (p[3] == 0) { o[0] = o[1] = o[2] = 0.0f; continue; }
            float f = std::ldexp(1.0f, (int)p[3] - (128 + 8));
            o[0] = p[0] * f; o[1] = p[1] * f; o[2] = p[2] * f;
        }
    }
    std::fclose(fp);
    return true;
}

// 32-bit BMP; row 0 of the image (the bottom row, TracingDetail.h:22-23) is
// written first, which is how a bottom-up BMP stores an upright picture.
bool write_bmp_rgba(const std::string& path, const uint8_t* rgba, uint32_t w, uint32_t h, bool flip, std::string& err) {
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) { err = "cannot write " + path; return false; }
    uint32_t row = w * 4, data = row * h, off = 14 + 40;
    uint8_t hdr[54] = {0};
    hdr[0] = 'B'; hdr[1] = 'M';
    auto put32 = [&](int at, uint32_t v) { for (int k = 0; k < 4; ++k) hdr[at + k] = (uint8_t)(v >> (8 * k)); };
    put32(2, off + data);
    put32(10, off);
    put32(14, 40);
    put32(18, w);
    put32(22, h);
    hdr[26] = 1;
    hdr[28] = 32;
    put32(34, data);
    std::fwrite(hdr, 1, 54, fp);
    std::vector<uint8_t> line(row);
    for (uint32_t yy = 0; yy < h; ++yy) {
        uint32_t y = flip ? h - 1 - yy : yy;
        const uint8_t* src = rgba + (size_t)y * row;
        for (uint32_t x = 0; x < w; ++x) {  // BGRA
            line[4 * x + 0] = src[4 * x + 2];
            line[4 * x + 1] = src[4 * x + 1];
            line[4 * x + 2] = src[4 * x + 0];
            line[4 * x + 3] = src[4 * x + 3];
        }
        std::fwrite(line.data(), 1, row, fp);
    }
    std::fclose(fp);
    return true;
}

// Portable float map, little endian (scale -1), rows bottom to top.
bool write_pfm(const std::string& path, const float* rgb, uint32_t w, uint32_t h, std::string& err) {
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) { err = "cannot write " + path; return false; }
    std::fprintf(fp, "PF\n%u %u\n-1.0\n", w, h);
    std::fwrite(rgb, sizeof(float), (size_t)w * h * 3, fp);
    std::fclose(fp);
    return true;
}

bool read_pfm(const std::string& path, std::vector<float>& rgb, uint32_t& w, uint32_t& h, std::string& err) {
    FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) { err = "cannot open " + path; return false; }
    char magic[3] = {0};
    float scale = 0;
    if (std::fscanf(fp, "%2s %u %u %f", magic, &w, &h, &scale) != 4 || std::strcmp(magic, "PF") != 0 || scale >= 0) {
        std::fclose(fp);
        err = path + ": only little-endian colour PFM is supported";
        return false;
    }
    std::fgetc(fp);
    rgb.resize((size_t)w * h * 3);
    size_t n = std::fread(rgb.data(), sizeof(float), rgb.size(), fp);
    std::fclose(fp);
    if (n != rgb.size()) { err = path + ": truncated"; return false; }
    return true;
}

// ------------------------------------------------------------ HostScene ---
uint32_t HostScene::add_sphere(const float pos[3], float radius, const HMaterial& m) {
    HObject o;
    o.type = GEO_SPHERE;
    o.mat = m;
    std::memcpy(o.p0, pos, 12);
    o.radius = radius;
    o.finite_box = true;  // SphereDetail.h:16
    for (int k = 0; k < 3; ++k) { o.box_lo[k] = pos[k] - radius; o.box_hi[k] = pos[k] + radius; }
    objects.push_back(o);
    return (uint32_t)objects.size() - 1;
}

uint32_t HostScene::add_plane(const float pos[3], const float normal[3], const HMaterial& m) {
    HObject o;
    o.type = GEO_PLANE;
    o.mat = m;
    std::memcpy(o.p0, pos, 12);
    std::memcpy(o.p1, normal, 12);
    objects.push_back(o);
    return (uint32_t)objects.size() - 1;
}

uint32_t HostScene::add_quad(const float pos[3], const float normal[3], const float e1[3], const float e2[3],
                             const HMaterial& m) {
    HObject o;
    o.type = GEO_QUAD;
    o.mat = m;
    std::memcpy(o.p0, pos, 12);
    std::memcpy(o.p1, normal, 12);
    std::memcpy(o.p2, e1, 12);
    std::memcpy(o.p3, e2, 12);
    objects.push_back(o);
    return (uint32_t)objects.size() - 1;
}

uint32_t HostScene::add_triangle(const float v1[3], const float v2[3], const float v3[3], const HMaterial& m) {
    HObject o;
    o.type = GEO_TRIANGLE;
    o.mat = m;
    o.tri_begin = (uint32_t)(tri_verts.size() / 9);
    o.tri_count = 1;
    tri_verts.insert(tri_verts.end(), v1, v1 + 3);
    tri_verts.insert(tri_verts.end(), v2, v2 + 3);
    tri_verts.insert(tri_verts.end(), v3, v3 + 3);
    objects.push_back(o);
    return (uint32_t)objects.size() - 1;
}

uint32_t HostScene::add_mesh(const float* verts, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float pos[3],
                             const float scale[3], const HMaterial& m) {
    HObject o;
    o.type = GEO_MESH;
    o.mat = m;
    o.tri_begin = (uint32_t)(tri_verts.size() / 9);
    o.tri_count = ntris;
    o.finite_box = true;
    std::vector<float> tv((size_t)nverts * 3);
    for (int k = 0; k < 3; ++k) { o.box_lo[k] = INFINITY; o.box_hi[k] = -INFINITY; }
    for (uint32_t i = 0; i < nverts; ++i)
        for (int k = 0; k < 3; ++k) {
            float v = scale[k] * verts[3 * i + k] + pos[k];  // ObjLoader.cpp:37
            tv[3 * i + k] = v;
            o.box_hi[k] = v > o.box_hi[k] ? v : o.box_hi[k];
            o.box_lo[k] = v < o.box_lo[k] ? v : o.box_lo[k];
        }
    // grow geometrically: an exact-size reserve per mesh would copy the whole
    // vertex array on every add (quadratic in the number of meshes)
    const size_t need = tri_verts.size() + (size_t)ntris * 9;
    if (tri_verts.capacity() < need) tri_verts.reserve(std::max(need, 2 * tri_verts.capacity()));
    for (uint32_t t = 0; t < ntris; ++t)
        for (int c = 0; c < 3; ++c) {
            const float* v = &tv[(size_t)idx[3 * t + c] * 3];
            tri_verts.insert(tri_verts.end(), v, v + 3);
        }
    objects.push_back(o);
    return (uint32_t)objects.size() - 1;
}

}  // namespace cupbr_b200
