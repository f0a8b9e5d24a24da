// pt_workloads.cpp — benchmark scenes and host ray generators (host C++17).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include "pt_exact.h"
#include "pt_host.h"
#include "pt_api_common.h"
#include "../../include/pt_workloads.h"


namespace ptb {
namespace {

// splitmix64: scene-generation random numbers (host only).
struct Mix {
    uint64_t s;
    explicit Mix(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return double(next() >> 11) * 0x1p-53; }
};

pt_vec3 v(float x, float y, float z) { return {x, y, z}; }
pt_triangle tri(pt_vec3 a, pt_vec3 b, pt_vec3 c, int32_t material) {
    pt_triangle t{};
    t.v0 = a; t.v1 = b; t.v2 = c;
    t.uv0 = v(0, 0, 0); t.uv1 = v(1, 0, 0); t.uv2 = v(0, 1, 0);   // triangle's default UVs
    t.material_id = material; t.smooth = 0;
    return t;
}
// quad p, p+a, p+a+b, p+b as two triangles; geometric normal along a x b
void quad(std::vector<pt_triangle> &out, pt_vec3 p, pt_vec3 a, pt_vec3 b, int32_t material) {
    pt_vec3 pa = v(p.x + a.x, p.y + a.y, p.z + a.z);
    pt_vec3 pab = v(pa.x + b.x, pa.y + b.y, pa.z + b.z);
    pt_vec3 pb = v(p.x + b.x, p.y + b.y, p.z + b.z);
    out.push_back(tri(p, pa, pab, material));
    out.push_back(tri(p, pab, pb, material));
}
int32_t constant_texture(FlatScene &s, pt_vec3 color) {
    pt_texture t{};
    t.color = color; t.scale = v(1, 1, 0); t.offset = v(0, 0, 0);
    t.type = PT_TEX_CONSTANT; t.image_id = -1; t.clamp = 1;   // flat_exporter's defaults (flat_export.h:39)
    s.textures.push_back(t);
    return int32_t(s.textures.size() - 1);
}
int32_t lambertian(FlatScene &s, pt_vec3 albedo) {
    pt_material m{};
    m.albedo = v(0, 0, 0); m.fuzz = 0; m.ref_idx = 1; m.type = PT_DIFFUSE; m.texture_id = constant_texture(s, albedo);
    s.materials.push_back(m);
    return int32_t(s.materials.size() - 1);
}
int32_t light(FlatScene &s, pt_vec3 radiance) {
    pt_material m{};
    m.albedo = v(0, 0, 0); m.fuzz = 0; m.ref_idx = 1; m.type = PT_LIGHT; m.texture_id = constant_texture(s, radiance);
    s.materials.push_back(m);
    return int32_t(s.materials.size() - 1);
}
int32_t metal(FlatScene &s, pt_vec3 albedo, float fuzz) {
    pt_material m{};
    m.albedo = albedo; m.fuzz = fuzz < 1 ? fuzz : 1; m.ref_idx = 1; m.type = PT_METAL; m.texture_id = -1;   // metal clamps fuzz (material.h:79-85)
    s.materials.push_back(m);
    return int32_t(s.materials.size() - 1);
}
int32_t glass(FlatScene &s, float ior) {
    pt_material m{};
    m.albedo = v(0, 0, 0); m.fuzz = 0; m.ref_idx = ior; m.type = PT_GLASS; m.texture_id = -1;
    s.materials.push_back(m);
    return int32_t(s.materials.size() - 1);
}

// Lattice value noise in [-1, 1], trilinear with smoothstep weights.
float lattice(int x, int y, int z, uint64_t seed) {
    uint64_t h = seed ^ (uint64_t(uint32_t(x)) * 0x8DA6B343ull) ^ (uint64_t(uint32_t(y)) * 0xD8163841ull) ^
                 (uint64_t(uint32_t(z)) * 0xCB1AB31Full);
    Mix m(h);
    return float(m.uniform() * 2.0 - 1.0);
}
float value_noise(double x, double y, double z, uint64_t seed) {
    int ix = int(std::floor(x)), iy = int(std::floor(y)), iz = int(std::floor(z));
    double fx = x - ix, fy = y - iy, fz = z - iz;
    auto sm = [](double t) { return t * t * (3 - 2 * t); };
    double wx = sm(fx), wy = sm(fy), wz = sm(fz);
    double r = 0;
    for(int dz = 0; dz < 2; dz++)
        for(int dy = 0; dy < 2; dy++)
            for(int dx = 0; dx < 2; dx++) {
                double w = (dx ? wx : 1 - wx) * (dy ? wy : 1 - wy) * (dz ? wz : 1 - wz);
                r += w * lattice(ix + dx, iy + dy, iz + dz, seed);
            }
    return float(r);
}

// Latitude-longitude sphere: pole fans plus (rings-2) quad bands = 2*segments*(rings-1)
// triangles, vertices displaced radially by value noise, wound outward.
void displaced_sphere(std::vector<pt_triangle> &out, double cx, double cy, double cz, double radius, int segments,
                      int rings, double amplitude, uint64_t seed, int32_t material) {
    auto vertex = [&](int ring, int seg) -> pt_vec3 {
        double theta = M_PI * double(ring) / rings, phi = 2 * M_PI * double(seg % segments) / segments;
        double dx = std::sin(theta) * std::cos(phi), dy = std::cos(theta), dz = std::sin(theta) * std::sin(phi);
        if(ring == 0) { dx = 0; dy = 1; dz = 0; }
        if(ring == rings) { dx = 0; dy = -1; dz = 0; }
        double n = value_noise(dx * 3 + 17.3, dy * 3 + 5.1, dz * 3 + 11.7, seed);
        double r = radius * (1 + amplitude * n);
        return v(float(cx + r * dx), float(cy + r * dy), float(cz + r * dz));
    };
    auto emit = [&](pt_vec3 a, pt_vec3 b, pt_vec3 c) {
        // orient outward: normal . (centroid - center) >= 0
        double e1[3] = {double(b.x) - a.x, double(b.y) - a.y, double(b.z) - a.z};
        double e2[3] = {double(c.x) - a.x, double(c.y) - a.y, double(c.z) - a.z};
        double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        double g[3] = {(double(a.x) + b.x + c.x) / 3 - cx, (double(a.y) + b.y + c.y) / 3 - cy, (double(a.z) + b.z + c.z) / 3 - cz};
        if(n[0] * g[0] + n[1] * g[1] + n[2] * g[2] < 0) std::swap(b, c);
        out.push_back(tri(a, b, c, material));
    };
    pt_vec3 north = vertex(0, 0), south = vertex(rings, 0);
    for(int j = 0; j < segments; j++) emit(north, vertex(1, j), vertex(1, j + 1));
    for(int i = 1; i < rings - 1; i++)
        for(int j = 0; j < segments; j++) {
            pt_vec3 a = vertex(i, j), b = vertex(i, j + 1), c = vertex(i + 1, j), d = vertex(i + 1, j + 1);
            emit(a, c, d);
            emit(a, d, b);
        }
    for(int j = 0; j < segments; j++) emit(south, vertex(rings - 1, j + 1), vertex(rings - 1, j));
}

double triangle_area(const pt_triangle &t) {
    double e1[3] = {double(t.v1.x) - t.v0.x, double(t.v1.y) - t.v0.y, double(t.v1.z) - t.v0.z};
    double e2[3] = {double(t.v2.x) - t.v0.x, double(t.v2.y) - t.v0.y, double(t.v2.z) - t.v0.z};
    double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    return 0.5 * std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
}

} // namespace
} // namespace ptb

using namespace ptb;

extern "C" {

pt_status pt_flat_from_desc(const pt_scene_desc *d, pt_flat **out) {
    return guard([&]() {
        if(!d || !out) throw Error(PT_INVALID_ARGUMENT, "null argument");
        auto h = new pt_flat;
        FlatScene &s = h->scene;
        s.triangles.assign(d->triangles, d->triangles + d->triangle_count);
        s.spheres.assign(d->spheres, d->spheres + d->sphere_count);
        s.nodes.assign(d->nodes, d->nodes + d->node_count);
        s.materials.assign(d->materials, d->materials + d->material_count);
        s.textures.assign(d->textures, d->textures + d->texture_count);
        s.pixels.assign(d->pixels, d->pixels + d->pixel_bytes);
        s.root = d->root; s.max_depth = d->max_depth;
        *out = h;
    });
}

pt_status pt_flat_build_bvh(pt_flat *scene, int threads) {
    return guard([&]() {
        if(!scene) throw Error(PT_INVALID_ARGUMENT, "null scene");
        build_sah(scene->scene, threads);
    });
}

pt_status pt_flat_desc(const pt_flat *scene, pt_scene_desc *desc) {
    return guard([&]() {
        if(!scene || !desc) throw Error(PT_INVALID_ARGUMENT, "null argument");
        *desc = scene->scene.desc();
    });
}

pt_status pt_flat_destroy(pt_flat *scene) { delete scene; return PT_OK; }

// camera::camera, src/core/camera.h:16-43, then flatten_camera (src/flat/flat_export.h:127-129)
pt_status pt_make_camera(const float lookfrom[3], const float lookat[3], const float vup[3], float vfov,
                         float aspect, float aperture, float focus_dist, float time0, float time1, pt_camera *out) {
    return guard([&]() {
        if(!out) throw Error(PT_INVALID_ARGUMENT, "null camera");
        float lens_radius = aperture / 2;
        float theta = float(vfov * M_PI / 180);
        float half_height = tanf(theta / 2);
        float half_width = aspect * half_height;
        f3 origin = mk(lookfrom[0], lookfrom[1], lookfrom[2]);
        f3 w = unit(origin - mk(lookat[0], lookat[1], lookat[2]));
        f3 u = unit(cross(mk(vup[0], vup[1], vup[2]), w));
        f3 vv = cross(w, u);
        f3 llc = origin - half_width * focus_dist * u - half_height * focus_dist * vv - focus_dist * w;
        out->origin = pv(origin);
        out->lower_left_corner = pv(llc);
        out->horizontal = pv(2 * half_width * focus_dist * u);
        out->vertical = pv(2 * half_height * focus_dist * vv);
        out->u = pv(u); out->v = pv(vv);
        out->lens_radius = lens_radius; out->time0 = time0; out->time1 = time1;
    });
}

pt_status pt_workload_cornell(int width, int height, pt_flat **out, pt_camera *camera) {
    return guard([&]() {
        if(!out || width <= 0 || height <= 0) throw Error(PT_INVALID_ARGUMENT, "invalid cornell arguments");
        auto h = new pt_flat;
        FlatScene &s = h->scene;
        int32_t white = lambertian(s, v(0.73f, 0.73f, 0.73f));
        int32_t red = lambertian(s, v(0.65f, 0.05f, 0.05f));
        int32_t green = lambertian(s, v(0.12f, 0.45f, 0.15f));
        int32_t lamp = light(s, v(15, 15, 15));
        int32_t mirror = metal(s, v(0.8f, 0.85f, 0.9f), 0.1f);
        int32_t clear = glass(s, 1.5f);
        const float D = 2.0f;                       // box depth; width and height are 1
        const float lx0 = 0.435f, lx1 = 0.565f;    // 0.13 wide
        const float lz0 = 0.945f, lz1 = 1.055f;    // 0.11 deep
        auto &T = s.triangles;
        quad(T, v(0, 0, 0), v(0, 0, D), v(1, 0, 0), white);                        // floor (+y)
        quad(T, v(0, 1, 0), v(1, 0, 0), v(0, 0, lz0), white);                      // ceiling pieces (-y)
        quad(T, v(0, 1, lz1), v(1, 0, 0), v(0, 0, D - lz1), white);
        quad(T, v(0, 1, lz0), v(lx0, 0, 0), v(0, 0, lz1 - lz0), white);
        quad(T, v(lx1, 1, lz0), v(1 - lx1, 0, 0), v(0, 0, lz1 - lz0), white);
        quad(T, v(lx0, 1, lz0), v(lx1 - lx0, 0, 0), v(0, 0, lz1 - lz0), lamp);     // emitter (-y)
        quad(T, v(0, 0, 0), v(1, 0, 0), v(0, 1, 0), white);                        // back (+z)
        quad(T, v(0, 0, D), v(0, 1, 0), v(1, 0, 0), white);                        // front (-z)
        quad(T, v(0, 0, 0), v(0, 1, 0), v(0, 0, D), red);                          // left (+x)
        quad(T, v(1, 0, 0), v(0, 0, D), v(0, 1, 0), green);                        // right (-x)
        s.spheres.push_back({v(0.3f, 0.18f, 0.55f), 0.18f, white});
        s.spheres.push_back({v(0.72f, 0.16f, 0.75f), 0.16f, mirror});
        s.spheres.push_back({v(0.5f, 0.15f, 1.15f), 0.15f, clear});
        build_sah(s, 1);
        if(camera) {
            float from[3] = {0.5f, 0.5f, 1.95f}, at[3] = {0.5f, 0.45f, 0.0f}, up[3] = {0, 1, 0};
            pt_status st = pt_make_camera(from, at, up, 40, float(width) / height, 0, 1.95f, 0, 1, camera);
            if(st != PT_OK) throw Error(st, pt_last_error());
        }
        *out = h;
    });
}

void pt_procedural_defaults(pt_procedural_params *p) {
    if(!p) return;
    std::memset(p, 0, sizeof *p);
    p->sphere_count = 16; p->segments = 256; p->rings = 129;
    p->box_size = 10; p->displacement = 0.05f; p->radius_min = 0.6f; p->radius_max = 1.2f;
    p->floor = 1; p->light_fraction = 0.005f; p->light_radiance = 40;
    p->metal_fraction = 0.2f; p->glass_fraction = 0.1f; p->seed = 1;
    p->random_triangles = 0; p->soup_edge_min = 1e-3f; p->soup_edge_max = 1e-2f;
}

pt_status pt_workload_procedural(const pt_procedural_params *p, int width, int height, pt_flat **out, pt_camera *camera) {
    return guard([&]() {
        if(!p || !out || width <= 0 || height <= 0 || p->sphere_count < 0 || p->segments < 3 || p->rings < 3 ||
           !(p->box_size > 0) || p->random_triangles < 0)
            throw Error(PT_INVALID_ARGUMENT, "invalid procedural scene parameters");
        auto h = new pt_flat;
        FlatScene &s = h->scene;
        Mix rng(p->seed * 0x2545F4914F6CDD1Dull + 1);
        const double B = p->box_size;
        size_t per = size_t(2) * size_t(p->segments) * size_t(p->rings - 1);
        s.triangles.reserve(per * size_t(p->sphere_count) + size_t(p->random_triangles) + 4);
        for(int i = 0; i < p->sphere_count; i++) {
            double cx = rng.uniform() * B, cy = rng.uniform() * B, cz = rng.uniform() * B;
            double radius = p->radius_min + rng.uniform() * (p->radius_max - p->radius_min);
            double kind = rng.uniform();
            pt_vec3 albedo = v(float(0.2 + 0.6 * rng.uniform()), float(0.2 + 0.6 * rng.uniform()), float(0.2 + 0.6 * rng.uniform()));
            float fuzz = float(0.3 * rng.uniform());
            uint64_t noise_seed = rng.next();
            int32_t m;
            if(kind < p->metal_fraction) m = metal(s, albedo, fuzz);
            else if(kind < p->metal_fraction + p->glass_fraction) m = glass(s, 1.5f);
            else m = lambertian(s, albedo);
            displaced_sphere(s.triangles, cx, cy, cz, radius, p->segments, p->rings, p->displacement, noise_seed, m);
        }
        if(p->random_triangles > 0) {
            int32_t grey = lambertian(s, v(0.6f, 0.6f, 0.6f));
            for(int i = 0; i < p->random_triangles; i++) {
                double c[3] = {rng.uniform() * B, rng.uniform() * B, rng.uniform() * B};
                pt_vec3 q[3];
                q[0] = v(float(c[0]), float(c[1]), float(c[2]));
                for(int k = 1; k < 3; k++) {
                    double len = p->soup_edge_min + rng.uniform() * (p->soup_edge_max - p->soup_edge_min);
                    double z = 2 * rng.uniform() - 1, a = 2 * M_PI * rng.uniform(), r = std::sqrt(std::max(0.0, 1 - z * z));
                    q[k] = v(float(c[0] + len * r * std::cos(a)), float(c[1] + len * z), float(c[2] + len * r * std::sin(a)));
                }
                s.triangles.push_back(tri(q[0], q[1], q[2], grey));
            }
        }
        if(p->floor) {
            int32_t ground = lambertian(s, v(0.5f, 0.5f, 0.5f));
            float lo = float(-0.5 * B), span = float(2 * B), y = float(-0.05 * B);
            quad(s.triangles, v(lo, y, lo), v(0, 0, span), v(span, 0, 0), ground);   // +y
        }
        if(p->light_fraction > 0) {
            double area = 0;
            for(const auto &t : s.triangles) area += triangle_area(t);
            double side = std::sqrt(p->light_fraction * area / (1 - p->light_fraction));
            int32_t lamp = light(s, v(p->light_radiance, p->light_radiance, p->light_radiance));
            float y = float(1.2 * B), x0 = float(0.5 * B - side / 2), z0 = float(0.5 * B - side / 2);
            quad(s.triangles, v(x0, y, z0), v(float(side), 0, 0), v(0, 0, float(side)), lamp);   // -y
        }
        if(p->gpu_bvh) build_lbvh(s); else build_sah(s, 0);
        if(camera) {
            float from[3] = {float(0.5 * B), float(0.75 * B), float(-1.1 * B)};
            float at[3] = {float(0.5 * B), float(0.35 * B), float(0.5 * B)}, up[3] = {0, 1, 0};
            float focus = std::sqrt((from[1] - at[1]) * (from[1] - at[1]) + (from[2] - at[2]) * (from[2] - at[2]));
            pt_status st = pt_make_camera(from, at, up, 40, float(width) / height, 0, focus, 0, 1, camera);
            if(st != PT_OK) throw Error(st, pt_last_error());
        }
        *out = h;
    });
}

pt_status pt_rays_camera(const pt_camera *camera, int width, int height, uint64_t seed, uint64_t first,
                         size_t count, pt_ray *rays) {
    return guard([&]() {
        if(!camera || (count && !rays) || width <= 0 || height <= 0) throw Error(PT_INVALID_ARGUMENT, "invalid camera ray arguments");
        uint64_t pixels = uint64_t(width) * uint64_t(height);
        for(size_t k = 0; k < count; k++) {
            uint64_t index = first + k;
            uint64_t pixel = index % pixels;
            int x = int(pixel % uint64_t(width)), y = int(pixel / uint64_t(width));
            Pcg r; r.seed(seed, index);
            float u = (x + r.uniform()) / float(width);
            float vv = (y + r.uniform()) / float(height);
            camera_ray(*camera, u, vv, r, rays[k]);
        }
    });
}

// The camera rays of pt_rays_camera with the given ray indices (index[k] in place of first + k).
pt_status pt_rays_camera_at(const pt_camera *camera, int width, int height, uint64_t seed, const uint64_t *index,
                            size_t count, pt_ray *rays) {
    return guard([&]() {
        if(!camera || (count && (!rays || !index)) || width <= 0 || height <= 0)
            throw Error(PT_INVALID_ARGUMENT, "invalid camera ray arguments");
        for(size_t k = 0; k < count; k++) {
            pt_status st = pt_rays_camera(camera, width, height, seed, index[k], 1, rays + k);
            if(st != PT_OK) throw Error(st, pt_last_error());
        }
    });
}

} // extern "C"


extern "C" pt_status pt_rays_surface(const pt_flat *scene, uint64_t seed, uint64_t first, size_t count,
                                     pt_ray *rays, float *shadow_tmax, int threads) {
    return guard([&]() {
        if(!scene || (count && !rays)) throw Error(PT_INVALID_ARGUMENT, "invalid surface ray arguments");
        const auto &T = scene->scene.triangles;
        if(T.empty()) throw Error(PT_INVALID_ARGUMENT, "surface rays need triangles");
        uint64_t ntri = T.size();
        int nt = threads > 0 ? threads : hardware_threads();
        if(size_t(nt) > count / 4096 + 1) nt = int(count / 4096 + 1);
        std::vector<std::thread> pool;
        for(int t = 0; t < nt; t++) {
            size_t b = count * size_t(t) / size_t(nt), e = count * size_t(t + 1) / size_t(nt);
            pool.emplace_back([&, b, e]() {
                for(size_t k = b; k < e; k++)
                    surface_ray(T.data(), ntri, seed, first + k, shadow_tmax != nullptr, rays[k], shadow_tmax ? shadow_tmax + k : nullptr);
            });
        }
        for(auto &th : pool) th.join();
    });
}

static void bounce_rays_host(const pt_flat *scene, const pt_ray *primary, const pt_hit *hits, size_t count, uint64_t seed,
                             uint64_t first, const uint64_t *streams, pt_ray *rays, int threads) {
    if(!scene || (count && (!primary || !hits || !rays))) throw Error(PT_INVALID_ARGUMENT, "invalid bounce ray arguments");
    const auto &T = scene->scene.triangles;
    const auto &S = scene->scene.spheres;
    if(T.empty()) throw Error(PT_INVALID_ARGUMENT, "bounce rays need triangles");
    for(size_t k = 0; k < count; k++) {
        const pt_hit &h = hits[k];
        if((h.primitive_type == PT_TRIANGLE && (h.primitive_id < 0 || size_t(h.primitive_id) >= T.size())) ||
           (h.primitive_type == PT_SPHERE && (h.primitive_id < 0 || size_t(h.primitive_id) >= S.size())))
            throw Error(PT_INVALID_ARGUMENT, "hit refers to a primitive outside the scene");
    }
    int nt = threads > 0 ? threads : hardware_threads();
    if(size_t(nt) > count / 4096 + 1) nt = int(count / 4096 + 1);
    std::vector<std::thread> pool;
    for(int t = 0; t < nt; t++) {
        size_t b = count * size_t(t) / size_t(nt), e = count * size_t(t + 1) / size_t(nt);
        pool.emplace_back([&, b, e]() {
            for(size_t k = b; k < e; k++)
                bounce_ray(T.data(), T.size(), S.data(), primary[k], hits[k], seed, streams ? streams[k] : first + k, rays[k]);
        });
    }
    for(auto &th : pool) th.join();
}

extern "C" pt_status pt_rays_bounce(const pt_flat *scene, const pt_ray *primary, const pt_hit *hits, size_t count,
                                    uint64_t seed, uint64_t first, pt_ray *rays, int threads) {
    return guard([&]() { bounce_rays_host(scene, primary, hits, count, seed, first, nullptr, rays, threads); });
}

extern "C" pt_status pt_rays_bounce_at(const pt_flat *scene, const pt_ray *primary, const pt_hit *hits, size_t count,
                                       uint64_t seed, const uint64_t *streams, pt_ray *rays, int threads) {
    return guard([&]() {
        if(count && !streams) throw Error(PT_INVALID_ARGUMENT, "null stream indices");
        bounce_rays_host(scene, primary, hits, count, seed, 0, streams, rays, threads);
    });
}
