// pt_obj.cpp — OBJ/MTL import and the reference's preview stage, producing a flat scene.
//
// Follows the reference's import (src/scene/obj_loader.h:116-237) and stage
// (src/scene/obj_scene.h:10-31):
//   * OBJ text as the reference's vendored tinyobjloader reads it (pinned in the reference's
//     third_party/tinyobjloader): numbers via its decimal reader (reproduced below so that
//     positions are bit-identical), 1-based / negative indices, quads split along the shorter
//     diagonal, larger polygons by its ear clipping in the polygon's dominant plane;
//   * MTL: Kd/Ks/Ke/Ni/illum/d/Ns/Pr/Pm and map_* with -s/-o/-clamp; material i gets slot i+1
//     after a grey fallback (0.7); emission > 0 -> light, illum 4/6/7/9 -> glass (Ni),
//     illum 3/5/8 -> mirror metal (Ks, fuzz 0), else Lambertian with Kd (clamped to [0,1]),
//     textured when map_Kd is set (image tinted by Kd, UV scale/offset/clamp);
//   * per triangle: unit normals when all three are usable (smooth), UVs when all three are
//     present (else (0,0), (1,0), (0,1)), degenerate triangles skipped, the mesh transform
//     (scale, X/Y/Z rotation in degrees, translation; normals by the inverse scale, mirrored
//     winding when an odd number of scales is negative, src/transforms/mesh_transform.h:10-80);
//   * stage: camera at 40 degrees framing the mesh bounds, a ground sphere of radius 100 r
//     (albedo 0.55) below and an emitting sphere of radius 1.5 r (radiance 3).
// The BVH is this library's binned SAH, so primitive ids differ from the reference's
// (its tree comes from a drand48 random-axis split); everything a shaded render reads is equal.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include "pt_api_common.h"
#include "pt_exact.h"
#include "pt_host.h"
#include "pt_image.h"
#include "../../include/pt_workloads.h"

using namespace ptb;

namespace {

// ---- tinyobjloader's decimal reader: digits into a double mantissa, fraction digits scaled
// by 10^-k (a table of powers for the first seven), exponent applied as ldexp(m * 5^e, e).
bool read_decimal(const char *s, const char *end, double &out) {
    if (s >= end) return false;
    double mantissa = 0.0;
    int exponent = 0;
    char sign = '+', exp_sign = '+';
    const char *c = s;
    bool leading_dot = false;
    if (*c == '+' || *c == '-') {
        sign = *c++;
        if (c != end && *c == '.') leading_dot = true;
    } else if (*c >= '0' && *c <= '9') {
    } else if (*c == '.') {
        leading_dot = true;
    } else {
        return false;
    }
    int count = 0;
    if (!leading_dot) {
        while (c != end && *c >= '0' && *c <= '9') { mantissa = mantissa * 10 + (*c - '0'); c++; count++; }
        if (count == 0) return false;
    }
    if (c != end) {
        bool exp_next = false;
        if (*c == '.') {
            c++;
            static const double table[] = {1.0, 0.1, 0.01, 0.001, 0.0001, 0.00001, 0.000001, 0.0000001};
            int k = 1;
            while (c != end && *c >= '0' && *c <= '9') {
                mantissa += (*c - '0') * (k < 8 ? table[k] : std::pow(10.0, -k));
                k++; c++;
            }
            exp_next = c != end;
        } else if (*c == 'e' || *c == 'E') {
            exp_next = true;
        }
        if (exp_next && (*c == 'e' || *c == 'E')) {
            c++;
            if (c != end && (*c == '+' || *c == '-')) exp_sign = *c++;
            else if (!(c != end && *c >= '0' && *c <= '9')) return false;
            count = 0;
            while (c != end && *c >= '0' && *c <= '9') {
                if (exponent > 2147483647 / 10) return false;
                exponent = exponent * 10 + (*c - '0');
                c++; count++;
            }
            if (exp_sign == '-') exponent = -exponent;
            if (count == 0) return false;
        }
    }
    out = (sign == '+' ? 1 : -1) * (exponent ? std::ldexp(mantissa * std::pow(5.0, exponent), exponent) : mantissa);
    return true;
}

// A cursor over one line; tokens are separated by spaces and tabs.
struct Cursor {
    const char *p, *e;
    void skip() { while (p < e && (*p == ' ' || *p == '\t')) p++; }
    std::pair<const char *, const char *> token() {
        skip();
        const char *b = p;
        while (p < e && *p != ' ' && *p != '\t' && *p != '\r') p++;
        return {b, p};
    }
    float real(double fallback = 0.0) {
        auto t = token();
        double v = fallback;
        read_decimal(t.first, t.second, v);
        return float(v);
    }
    bool at_end() { skip(); return p >= e; }
    std::string rest() { skip(); return std::string(p, e); }
};

struct MtlTexOpt { float scale[3] = {1, 1, 1}, offset[3] = {0, 0, 0}; bool clamp = false; };
struct MtlMaterial {
    std::string name, diffuse_tex, alpha_tex, bump_tex, normal_tex, emissive_tex;
    float ambient[3] = {0, 0, 0}, diffuse[3] = {0, 0, 0}, specular[3] = {0, 0, 0}, transmittance[3] = {0, 0, 0},
          emission[3] = {0, 0, 0};
    float ior = 1, dissolve = 1, shininess = 1, roughness = 0, metallic = 0;
    int illum = 0;
    MtlTexOpt diffuse_opt;
    std::filesystem::path directory;
};

// map_* value: options (-s u [v [w]], -o u [v [w]], -clamp on|off, others skipped), then the
// rest of the line is the file name (names may hold spaces).
std::string texture_name(Cursor c, MtlTexOpt *opt) {
    for (;;) {
        c.skip();
        if (c.p >= c.e) return "";
        auto starts = [&](const char *word) {
            size_t n = std::strlen(word);
            return size_t(c.e - c.p) > n && std::strncmp(c.p, word, n) == 0 && (c.p[n] == ' ' || c.p[n] == '\t');
        };
        auto reals = [&](int n, float *out, bool store) {
            c.p += 3;
            for (int k = 0; k < n; k++) { float v = c.real(0.0); if (store) out[k] = v; }
        };
        if (starts("-clamp")) {
            c.p += 7;
            auto t = c.token();
            bool on = true;
            if (t.second - t.first >= 2 && std::strncmp(t.first, "on", 2) == 0) on = true;
            else if (t.second - t.first >= 3 && std::strncmp(t.first, "off", 3) == 0) on = false;
            if (opt) opt->clamp = on;
        } else if (starts("-s")) { reals(3, opt ? opt->scale : nullptr, opt != nullptr);
        } else if (starts("-o")) { reals(3, opt ? opt->offset : nullptr, opt != nullptr);
        } else if (starts("-t")) { float t3[3]; reals(3, t3, false);
        } else if (starts("-bm")) { c.p += 4; c.real();
        } else if (starts("-blendu") || starts("-blendv") || starts("-cc")) {
            while (c.p < c.e && *c.p != ' ' && *c.p != '\t') c.p++;
            c.token();
        } else if (starts("-mm")) { c.p += 4; c.real(); c.real(1.0);
        } else if (starts("-boost")) { c.p += 7; c.real();
        } else if (starts("-texres") || starts("-type") || starts("-imfchan") || starts("-colorspace")) {
            while (c.p < c.e && *c.p != ' ' && *c.p != '\t') c.p++;
            c.token();
        } else {
            return std::string(c.p, c.e);
        }
    }
}

std::vector<std::string> lines_of(const std::string &path, bool &ok) {
    std::ifstream in(path, std::ios::binary);
    ok = bool(in);
    std::vector<std::string> lines;
    std::string line;
    while (ok && std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        lines.push_back(line);
    }
    return lines;
}

void load_mtl(const std::filesystem::path &file, std::vector<MtlMaterial> &out, std::map<std::string, int> &names) {
    bool ok;
    auto lines = lines_of(file.string(), ok);
    if (!ok) throw Error(PT_INVALID_ARGUMENT, "could not load MTL: " + file.string() +
                         "\nCheck the OBJ mtllib filename and keep the referenced MTL beside the OBJ (or at that relative path).");
    MtlMaterial m;
    bool have = false;
    auto flush = [&]() {
        if (!have) return;
        m.directory = file.parent_path();
        names[m.name] = int(out.size());
        out.push_back(m);
    };
    for (const std::string &text : lines) {
        Cursor c{text.data(), text.data() + text.size()};
        c.skip();
        if (c.p >= c.e || *c.p == '#') continue;
        auto key = c.token();
        std::string k(key.first, key.second);
        auto three = [&](float *v) { v[0] = c.real(); v[1] = c.real(); v[2] = c.real(); };
        if (k == "newmtl") { flush(); m = MtlMaterial(); have = true; m.name = c.rest(); }
        else if (k == "Ka") three(m.ambient);
        else if (k == "Kd") three(m.diffuse);
        else if (k == "Ks") three(m.specular);
        else if (k == "Kt" || k == "Tf") three(m.transmittance);
        else if (k == "Ke") three(m.emission);
        else if (k == "Ni") m.ior = c.real();
        else if (k == "Ns") m.shininess = c.real();
        else if (k == "illum") { auto t = c.token(); m.illum = std::atoi(std::string(t.first, t.second).c_str()); }
        else if (k == "d") m.dissolve = c.real();
        else if (k == "Tr") m.dissolve = 1.0f - c.real();
        else if (k == "Pr") m.roughness = c.real();
        else if (k == "Pm") m.metallic = c.real();
        else if (k == "map_Kd") m.diffuse_tex = texture_name(c, &m.diffuse_opt);
        else if (k == "map_d") m.alpha_tex = texture_name(c, nullptr);
        else if (k == "map_bump" || k == "map_Bump" || k == "bump") m.bump_tex = texture_name(c, nullptr);
        else if (k == "norm" || k == "map_Kn") m.normal_tex = texture_name(c, nullptr);
        else if (k == "map_Ke") m.emissive_tex = texture_name(c, nullptr);
    }
    flush();
}

struct Corner { int v, vt, vn; };

// index as written -> 0-based (negative = relative to the count so far); 0 is an error
int fix_index(int idx, size_t count) {
    if (idx > 0) return idx - 1;
    if (idx < 0) return int(count) + idx;
    throw Error(PT_INVALID_ARGUMENT, "OBJ load failed: zero value for face index");
}

bool point_in_triangle(const float *vx, const float *vy, float tx, float ty) {
    bool inside = false;
    for (int i = 0, j = 2; i < 3; j = i++) {
        if (((vy[i] > ty) != (vy[j] > ty)) && (tx < (vx[j] - vx[i]) * (ty - vy[i]) / (vy[j] - vy[i]) + vx[i])) inside = !inside;
    }
    return inside;
}

// Triangulation of one face into `out` (corner triples), as the reference's loader does it.
void triangulate(const std::vector<Corner> &face, const std::vector<float> &v, std::vector<Corner> &out, std::string &warnings) {
    const size_t n = face.size();
    auto valid = [&](const Corner &k) { return size_t(3 * k.v + 2) < v.size() && k.v >= 0; };
    if (n < 3) { warnings += "Degenerated face found\n."; return; }
    if (n == 3) { out.insert(out.end(), face.begin(), face.end()); return; }
    if (n == 4) {
        for (const Corner &k : face) if (!valid(k)) { warnings += "Face with invalid vertex index found.\n"; return; }
        auto P = [&](int i, int a) { return v[size_t(face[i].v) * 3 + a]; };
        float e02[3], e13[3];
        for (int a = 0; a < 3; a++) { e02[a] = P(2, a) - P(0, a); e13[a] = P(3, a) - P(1, a); }
        float s02 = e02[0] * e02[0] + e02[1] * e02[1] + e02[2] * e02[2];
        float s13 = e13[0] * e13[0] + e13[1] * e13[1] + e13[2] * e13[2];
        if (s02 < s13) out.insert(out.end(), {face[0], face[1], face[2], face[0], face[2], face[3]});
        else out.insert(out.end(), {face[0], face[1], face[3], face[1], face[2], face[3]});
        return;
    }
    // dominant plane: from the first corner with a non-negligible cross product
    size_t axes[2] = {1, 2};
    for (size_t k = 0; k < n; k++) {
        const Corner &a = face[k % n], &b = face[(k + 1) % n], &c = face[(k + 2) % n];
        if (!valid(a) || !valid(b) || !valid(c)) continue;
        float e0[3], e1[3];
        for (int q = 0; q < 3; q++) { e0[q] = v[size_t(b.v) * 3 + q] - v[size_t(a.v) * 3 + q]; e1[q] = v[size_t(c.v) * 3 + q] - v[size_t(b.v) * 3 + q]; }
        float cx = std::fabs(e0[1] * e1[2] - e0[2] * e1[1]), cy = std::fabs(e0[2] * e1[0] - e0[0] * e1[2]),
              cz = std::fabs(e0[0] * e1[1] - e0[1] * e1[0]);
        const float eps = 1.1920929e-07f;
        if (cx > eps || cy > eps || cz > eps) {
            if (!(cx > cy && cx > cz)) {
                axes[0] = 0;
                if (cz > cx && cz > cy) axes[1] = 1;
            }
            break;
        }
    }
    std::vector<Corner> rem = face;
    size_t guess = 0, tries = n, previous = rem.size();
    auto coord = [&](const Corner &k, int a) -> float {
        size_t i = size_t(k.v) * 3 + axes[a];
        return (k.v >= 0 && i < v.size()) ? v[i] : 0.0f;
    };
    while (rem.size() > 3 && tries > 0) {
        const size_t m = rem.size();
        if (guess >= m) guess -= m;
        if (previous != m) { previous = m; tries = m; } else tries--;
        Corner ind[3];
        float vx[3], vy[3];
        for (int k = 0; k < 3; k++) { ind[k] = rem[(guess + k) % m]; vx[k] = coord(ind[k], 0); vy[k] = coord(ind[k], 1); }
        float e0x = vx[1] - vx[0], e0y = vy[1] - vy[0], e1x = vx[2] - vx[1], e1y = vy[2] - vy[1];
        float cross = e0x * e1y - e0y * e1x;
        float area = (vx[0] * vy[1] - vy[0] * vx[1]) * 0.5f;
        if (cross * area < 0.0f) { guess++; continue; }
        bool overlap = false;
        for (size_t o = 3; o < m; o++) {
            const Corner &k = rem[(guess + o) % m];
            size_t i0 = size_t(k.v) * 3 + axes[0], i1 = size_t(k.v) * 3 + axes[1];
            if (k.v < 0 || i0 >= v.size() || i1 >= v.size()) continue;
            if (point_in_triangle(vx, vy, v[i0], v[i1])) { overlap = true; break; }
        }
        if (overlap) { guess++; continue; }
        out.insert(out.end(), {ind[0], ind[1], ind[2]});
        rem.erase(rem.begin() + long((guess + 1) % m));
    }
    if (rem.size() == 3) out.insert(out.end(), {rem[0], rem[1], rem[2]});
}

f3 attribute(const std::vector<float> &values, int index, int width) {
    if (index < 0 || size_t(index) >= values.size() / size_t(width)) throw Error(PT_INVALID_ARGUMENT, "OBJ attribute index is out of range");
    size_t o = size_t(index) * size_t(width);
    f3 r = mk(values[o], values[o + 1], width == 3 ? values[o + 2] : 0.0f);
    if (!std::isfinite(r.x) || !std::isfinite(r.y) || !std::isfinite(r.z)) throw Error(PT_INVALID_ARGUMENT, "OBJ contains a non-finite attribute");
    return r;
}

f3 mtl_color(const float c[3], bool reflectance) {
    f3 v = mk(c[0], c[1], c[2]);
    if (!std::isfinite(v.x) || !std::isfinite(v.y) || !std::isfinite(v.z)) throw Error(PT_INVALID_ARGUMENT, "MTL contains a non-finite color");
    float *p[3] = {&v.x, &v.y, &v.z};
    for (float *x : p) { *x = std::fmax(0.0f, *x) == *x ? *x : 0.0f; if (*x < 0) *x = 0; if (reflectance && *x > 1) *x = 1; }
    return v;
}

// Scale, X/Y/Z rotations (degrees, angles reduced mod 360 in double), translation.
struct Transform {
    f3 factors, offset;
    float sine[3], cosine[3];
    bool unchanged = true, mirrored = false;
    Transform(const float s[3], const float r[3], const float t[3]) {
        factors = mk(s[0], s[1], s[2]);
        offset = mk(t[0], t[1], t[2]);
        for (int i = 0; i < 3; i++) {
            if (!std::isfinite(s[i]) || s[i] == 0 || !std::isfinite(r[i]) || !std::isfinite(t[i]))
                throw Error(PT_INVALID_ARGUMENT, "mesh transform requires finite values and nonzero scale");
            double angle = std::remainder(double(r[i]), 360.0) * 3.14159265358979323846 / 180.0;
            sine[i] = float(std::sin(angle));
            cosine[i] = float(std::cos(angle));
            if (s[i] != 1 || r[i] != 0 || t[i] != 0) unchanged = false;
            if (s[i] < 0) mirrored = !mirrored;
        }
    }
    f3 rotate(f3 v) const {
        v = mk(v.x, cosine[0] * v.y - sine[0] * v.z, sine[0] * v.y + cosine[0] * v.z);
        v = mk(cosine[1] * v.x + sine[1] * v.z, v.y, -sine[1] * v.x + cosine[1] * v.z);
        return mk(cosine[2] * v.x - sine[2] * v.y, sine[2] * v.x + cosine[2] * v.y, v.z);
    }
    f3 position(f3 p) const {
        f3 r = rotate(p * factors) + offset;
        if (!std::isfinite(r.x) || !std::isfinite(r.y) || !std::isfinite(r.z)) throw Error(PT_INVALID_ARGUMENT, "transformed position exceeds float range");
        return r;
    }
    f3 normal(f3 n) const {
        double x = double(n.x) / factors.x, y = double(n.y) / factors.y, z = double(n.z) / factors.z;
        double len = std::sqrt(x * x + y * y + z * z);
        if (!(len > 0) || !std::isfinite(len)) throw Error(PT_INVALID_ARGUMENT, "invalid transformed normal");
        return unit(rotate(mk(float(x / len), float(y / len), float(z / len))));
    }
    void apply(pt_triangle &t) const {
        if (unchanged) return;
        t.v0 = pv(position(mk(t.v0))); t.v1 = pv(position(mk(t.v1))); t.v2 = pv(position(mk(t.v2)));
        if (t.smooth) { t.n0 = pv(normal(mk(t.n0))); t.n1 = pv(normal(mk(t.n1))); t.n2 = pv(normal(mk(t.n2))); }
        if (mirrored) { std::swap(t.v1, t.v2); std::swap(t.n1, t.n2); std::swap(t.uv1, t.uv2); }
        float area = sqlen(cross(mk(t.v1) - mk(t.v0), mk(t.v2) - mk(t.v0)));
        if (!(area > 0) || !std::isfinite(area)) throw Error(PT_INVALID_ARGUMENT, "mesh transform collapses geometry or exceeds supported float range");
    }
};

std::filesystem::path asset_path(std::string p) {
    for (char &c : p) if (c == '\\') c = '/';
    return std::filesystem::path(p);
}

int32_t add_texture(FlatScene &s, const pt_texture &t) { s.textures.push_back(t); return int32_t(s.textures.size() - 1); }
pt_texture constant_record(f3 color) {
    pt_texture t{};
    t.color = pv(color); t.scale = pt_vec3{1, 1, 0}; t.offset = pt_vec3{0, 0, 0};
    t.type = PT_TEX_CONSTANT; t.image_id = -1; t.clamp = 1;
    return t;
}
int32_t add_material(FlatScene &s, int32_t type, f3 albedo, float fuzz, float ior, int32_t texture) {
    pt_material m{};
    m.albedo = pv(albedo); m.fuzz = fuzz; m.ref_idx = ior; m.type = type; m.texture_id = texture;
    s.materials.push_back(m);
    return int32_t(s.materials.size() - 1);
}

// OBJ + MTL -> triangles (appended to s.triangles) and materials/textures; returns the warnings.
std::string import_obj(const std::string &filename, const Transform &xf, FlatScene &s) {
    std::filesystem::path path = asset_path(filename);
    bool ok;
    auto lines = lines_of(path.string(), ok);
    if (!ok) throw Error(PT_INVALID_ARGUMENT, "could not load OBJ: " + filename);
    std::string warnings;
    std::vector<float> pos, tex, nrm;
    std::vector<MtlMaterial> mtl;
    std::map<std::string, int> names;
    struct Face { std::vector<Corner> corners; int material; };
    std::vector<Face> faces;
    std::vector<std::string> line_shapes;
    std::string shape_name;
    bool shape_has_lines = false;
    int current = -1;
    auto end_shape = [&]() { if (shape_has_lines) line_shapes.push_back(shape_name); shape_has_lines = false; };
    for (const std::string &text : lines) {
        Cursor c{text.data(), text.data() + text.size()};
        c.skip();
        if (c.p >= c.e || *c.p == '#') continue;
        auto key = c.token();
        std::string k(key.first, key.second);
        if (k == "v") { pos.push_back(c.real()); pos.push_back(c.real()); pos.push_back(c.real()); }
        else if (k == "vt") { tex.push_back(c.real()); tex.push_back(c.real()); }
        else if (k == "vn") { nrm.push_back(c.real()); nrm.push_back(c.real()); nrm.push_back(c.real()); }
        else if (k == "f") {
            Face f;
            f.material = current;
            while (!c.at_end()) {
                auto t = c.token();
                std::string tok(t.first, t.second);
                Corner k3{-1, -1, -1};
                int a = 0, b = 0, d = 0;
                size_t s1 = tok.find('/');
                a = std::atoi(tok.c_str());
                k3.v = fix_index(a, pos.size() / 3);
                if (s1 != std::string::npos) {
                    size_t s2 = tok.find('/', s1 + 1);
                    if (s2 == std::string::npos) { b = std::atoi(tok.c_str() + s1 + 1); k3.vt = fix_index(b, tex.size() / 2); }
                    else {
                        if (s2 > s1 + 1) { b = std::atoi(tok.c_str() + s1 + 1); k3.vt = fix_index(b, tex.size() / 2); }
                        d = std::atoi(tok.c_str() + s2 + 1);
                        k3.vn = fix_index(d, nrm.size() / 3);
                    }
                }
                f.corners.push_back(k3);
            }
            faces.push_back(std::move(f));
        } else if (k == "usemtl") {
            std::string name = c.rest();
            auto it = names.find(name);
            if (it == names.end()) { warnings += "material [ '" + name + "' ] not found in .mtl\n"; current = -1; }
            else current = it->second;
        } else if (k == "mtllib") {
            std::string rest = c.rest();
            std::istringstream files(rest);
            std::string one;
            bool loaded = false;
            while (files >> one && !loaded) { load_mtl(path.parent_path() / asset_path(one), mtl, names); loaded = true; }
        } else if (k == "o" || k == "g") {
            end_shape();
            shape_name = c.rest();
        } else if (k == "l" || k == "p") {
            shape_has_lines = true;
        }
    }
    end_shape();
    for (const std::string &name : line_shapes) warnings += "Ignoring OBJ lines/points in '" + name + "'.\n";

    // materials: slot 0 the grey fallback, MTL material i in slot i + 1
    std::vector<int32_t> slot;
    slot.push_back(add_material(s, PT_DIFFUSE, mk(0, 0, 0), 0, 1, add_texture(s, constant_record(mk(0.7f, 0.7f, 0.7f)))));
    std::map<std::string, int32_t> images;
    for (const MtlMaterial &m : mtl) {
        f3 diffuse = mtl_color(m.diffuse, true), emission = mtl_color(m.emission, false);
        bool glass = m.illum == 4 || m.illum == 6 || m.illum == 7 || m.illum == 9;
        bool mirror = m.illum == 3 || m.illum == 5 || m.illum == 8;
        if (sqlen(emission) > 0) {
            slot.push_back(add_material(s, PT_LIGHT, mk(0, 0, 0), 0, 1, add_texture(s, constant_record(emission))));
        } else if (glass) {
            if (!(m.ior > 0) || !std::isfinite(m.ior)) throw Error(PT_INVALID_ARGUMENT, "invalid MTL refractive index");
            slot.push_back(add_material(s, PT_GLASS, mk(0, 0, 0), 0, m.ior, -1));
        } else if (mirror) {
            slot.push_back(add_material(s, PT_METAL, mtl_color(m.specular, true), 0, 1, -1));
        } else if (m.diffuse_tex.empty()) {
            slot.push_back(add_material(s, PT_DIFFUSE, mk(0, 0, 0), 0, 1, add_texture(s, constant_record(diffuse))));
        } else {
            std::string file = (m.directory / asset_path(m.diffuse_tex)).lexically_normal().string();
            auto it = images.find(file);
            int32_t image;
            if (it != images.end()) image = it->second;
            else {
                Image img;
                std::string err;
                if (!load_image(file, img, err)) throw Error(PT_INVALID_ARGUMENT, "could not load texture: " + err);
                uint64_t bytes = uint64_t(img.width) * uint64_t(img.height) * 3;
                if (bytes + s.pixels.size() >= uint64_t(INT32_MAX)) throw Error(PT_INVALID_ARGUMENT, "flat image storage exceeds 32-bit offsets");
                pt_texture t = constant_record(mk(0, 0, 0));
                t.type = PT_TEX_IMAGE; t.width = img.width; t.height = img.height; t.byte_offset = int32_t(s.pixels.size());
                s.pixels.insert(s.pixels.end(), img.rgb.begin(), img.rgb.end());
                image = add_texture(s, t);
                images[file] = image;
            }
            pt_texture map = constant_record(diffuse);
            map.type = PT_TEX_MAP; map.image_id = image;
            map.scale = pt_vec3{m.diffuse_opt.scale[0], m.diffuse_opt.scale[1], 0};
            map.offset = pt_vec3{m.diffuse_opt.offset[0], m.diffuse_opt.offset[1], 0};
            map.clamp = m.diffuse_opt.clamp ? 1 : 0;
            if (!std::isfinite(map.scale.x) || !std::isfinite(map.scale.y) || !std::isfinite(map.offset.x) || !std::isfinite(map.offset.y))
                throw Error(PT_INVALID_ARGUMENT, "invalid MTL UV transform");
            slot.push_back(add_material(s, PT_DIFFUSE, mk(0, 0, 0), 0, 1, add_texture(s, map)));
        }
        if (m.dissolve != 1 || !m.alpha_tex.empty() || !m.bump_tex.empty() || !m.normal_tex.empty() || !m.emissive_tex.empty() ||
            m.metallic != 0 || m.roughness != 0 || m.shininess != 1 || m.specular[0] != 0 || m.specular[1] != 0 || m.specular[2] != 0)
            warnings += "MTL '" + m.name + "': simplified material mapping; see README for unsupported shading properties.\n";
    }

    size_t degenerate = 0, missing_uv = 0, flat = 0;
    const size_t first = s.triangles.size();
    std::vector<Corner> tri;
    for (const Face &f : faces) {
        tri.clear();
        triangulate(f.corners, pos, tri, warnings);
        for (size_t t = 0; t + 2 < tri.size(); t += 3) {
            f3 p[3], n[3], uv[3];
            bool has_n = true, has_uv = true;
            for (int k = 0; k < 3; k++) {
                const Corner &q = tri[t + size_t(k)];
                p[k] = attribute(pos, q.v, 3);
                if (q.vn < 0) has_n = false;
                else {
                    n[k] = attribute(nrm, q.vn, 3);
                    float len = length(n[k]);
                    if (!(len > 0) || !std::isfinite(len)) has_n = false;
                    else n[k] = div_assign(n[k], len);
                }
                if (q.vt < 0) has_uv = false;
                else uv[k] = attribute(tex, q.vt, 2);
            }
            float area2 = sqlen(cross(p[1] - p[0], p[2] - p[0]));
            if (!std::isfinite(area2)) throw Error(PT_INVALID_ARGUMENT, "OBJ geometry exceeds supported float range");
            if (!(area2 > 0)) { degenerate++; continue; }
            if (f.material < -1 || f.material >= int(mtl.size())) throw Error(PT_INVALID_ARGUMENT, "invalid OBJ material index");
            pt_triangle face{};
            face.v0 = pv(p[0]); face.v1 = pv(p[1]); face.v2 = pv(p[2]);
            face.material_id = slot[size_t(f.material + 1)];
            if (has_n) { face.smooth = 1; face.n0 = pv(n[0]); face.n1 = pv(n[1]); face.n2 = pv(n[2]); }
            else flat++;
            if (has_uv) { face.uv0 = pv(uv[0]); face.uv1 = pv(uv[1]); face.uv2 = pv(uv[2]); }
            else { missing_uv++; face.uv0 = pt_vec3{0, 0, 0}; face.uv1 = pt_vec3{1, 0, 0}; face.uv2 = pt_vec3{0, 1, 0}; }
            xf.apply(face);
            s.triangles.push_back(face);
        }
    }
    if (s.triangles.size() == first) throw Error(PT_INVALID_ARGUMENT, "OBJ contains no usable triangles: " + filename);
    if (degenerate) warnings += "Skipped " + std::to_string(degenerate) + " degenerate triangles.\n";
    if (flat) warnings += "Using face normals for " + std::to_string(flat) + " triangles without complete usable normals.\n";
    if (missing_uv) warnings += "Using canonical UVs for " + std::to_string(missing_uv) + " triangles without complete UVs.\n";
    return warnings;
}

} // namespace

extern "C" pt_status pt_workload_obj(const char *path, int width, int height, const float scale[3], const float rotate[3],
                                     const float translate[3], pt_flat **out, pt_camera *camera, char *warnings, size_t capacity) {
    return guard([&]() {
        if (!path || !out || width <= 0 || height <= 0) throw Error(PT_INVALID_ARGUMENT, "invalid OBJ scene arguments");
        *out = nullptr;
        if (!*path) throw Error(PT_INVALID_ARGUMENT, "OBJ filename must not be empty");
        const float one[3] = {1, 1, 1}, zero[3] = {0, 0, 0};
        Transform xf(scale ? scale : one, rotate ? rotate : zero, translate ? translate : zero);
        auto h = new pt_flat;
        try {
            FlatScene &s = h->scene;
            std::string warn = import_obj(path, xf, s);
            // the stage (src/scene/obj_scene.h:14-26): bounds of the padded triangle boxes
            const float inf = std::numeric_limits<float>::infinity();
            float lo[3] = {inf, inf, inf}, hi[3] = {-inf, -inf, -inf};
            for (const pt_triangle &t : s.triangles) {
                const float *v[3] = {&t.v0.x, &t.v1.x, &t.v2.x};
                for (int a = 0; a < 3; a++) {
                    float mn = std::fmin(v[0][a], std::fmin(v[1][a], v[2][a])), mx = std::fmax(v[0][a], std::fmax(v[1][a], v[2][a]));
                    lo[a] = std::fmin(lo[a], std::nextafter(mn - 0.0001f, -inf));
                    hi[a] = std::fmax(hi[a], std::nextafter(mx + 0.0001f, inf));
                }
            }
            f3 bmin = mk(lo[0], lo[1], lo[2]), bmax = mk(hi[0], hi[1], hi[2]);
            f3 lookat = 0.5f * bmin + 0.5f * bmax;
            float radius = std::fmax(0.01f, 0.5f * length(bmax - bmin));
            if (!std::isfinite(radius)) throw Error(PT_INVALID_ARGUMENT, "OBJ bounds exceed camera range");
            const float aspect = float(width) / float(height);
            float half_angle = float(std::atan(std::tan(20 * M_PI / 180) * double(std::fmin(1.0f, aspect))));
            // the reference's sin(half_angle) takes the float overload (its tan and atan take doubles)
            float focus = (1.2f * radius) / std::sin(half_angle);
            f3 lookfrom = lookat + focus * unit(mk(0.6f, 0.35f, 1.0f));
            int32_t floor_mat = add_material(s, PT_DIFFUSE, mk(0, 0, 0), 0, 1, add_texture(s, constant_record(mk(0.55f, 0.55f, 0.55f))));
            int32_t light_mat = add_material(s, PT_LIGHT, mk(0, 0, 0), 0, 1, add_texture(s, constant_record(mk(3, 3, 3))));
            pt_sphere ground{pt_vec3{lookat.x, bmin.y - 100 * radius, lookat.z}, 100 * radius, floor_mat};
            pt_sphere light{pv(lookat + radius * mk(-1, 3, 3)), 1.5f * radius, light_mat};
            s.spheres.push_back(ground);
            s.spheres.push_back(light);
            build_sah(s, 0);
            if (camera) {
                const float from[3] = {lookfrom.x, lookfrom.y, lookfrom.z}, at[3] = {lookat.x, lookat.y, lookat.z}, up[3] = {0, 1, 0};
                pt_status st = pt_make_camera(from, at, up, 40, aspect, 0, focus, 0, 1, camera);
                if (st != PT_OK) throw Error(st, pt_last_error());
            }
            if (warnings && capacity) {
                std::strncpy(warnings, warn.c_str(), capacity - 1);
                warnings[capacity - 1] = 0;
            }
        } catch (...) { delete h; throw; }
        *out = h;
    });
}
