// ref_shim.cpp — C entry points around the reference's OWN host code (TEST INFRASTRUCTURE ONLY).
//
// Compiled by oracle/Makefile against the reference's headers where they lie
// (AdmiralHeathCL/cuda-path-tracer: src/, tests/support/, third_party/) into
// oracle/_ref/libref_cpu.so.  Nothing here restates the reference: every answer comes from
// the reference's own functions (trace_world, trace_pixel_sample, scene_lights,
// validate_flat_scene, flatten_scene, obj_scene, bvh_node::hit, portable_renderer), driven
// through plain C signatures so the Python tests and the CPU baseline can call them.
#include <cstring>
#include <thread>
#include <vector>
#include <atomic>

#include "flat/flat_export.h"
#include "renderer/render_validation.h"
#include "renderer/transport.h"
#include "support/portable_renderer.h"
#include "display/display_pixels.h"
#include "../include/pt.h"

static_assert(sizeof(flat_triangle) == sizeof(pt_triangle), "triangle layout");
static_assert(sizeof(flat_sphere) == sizeof(pt_sphere), "sphere layout");
static_assert(sizeof(flat_node) == sizeof(pt_node), "node layout");
static_assert(sizeof(flat_material) == sizeof(pt_material), "material layout");
static_assert(sizeof(flat_texture) == sizeof(pt_texture), "texture layout");
static_assert(sizeof(flat_camera) == sizeof(pt_camera), "camera layout");
static_assert(sizeof(ray) == sizeof(pt_ray), "ray layout");
static_assert(sizeof(trace_result) == sizeof(pt_trace_result), "trace_result layout");
static_assert(sizeof(flat_light) == sizeof(pt_light), "light layout");
static_assert(sizeof(pixel_rng) == 16, "rng layout");

namespace {
flat_scene to_scene(const pt_scene_desc *d) {
    flat_scene s;
    auto tri = reinterpret_cast<const flat_triangle *>(d->triangles);
    auto sph = reinterpret_cast<const flat_sphere *>(d->spheres);
    auto nod = reinterpret_cast<const flat_node *>(d->nodes);
    auto mat = reinterpret_cast<const flat_material *>(d->materials);
    auto tex = reinterpret_cast<const flat_texture *>(d->textures);
    s.triangles.assign(tri, tri + d->triangle_count);
    s.spheres.assign(sph, sph + d->sphere_count);
    s.nodes.assign(nod, nod + d->node_count);
    s.materials.assign(mat, mat + d->material_count);
    s.textures.assign(tex, tex + d->texture_count);
    s.pixels.assign(d->pixels, d->pixels + d->pixel_bytes);
    s.root = d->root;
    s.max_depth = d->max_depth;
    return s;
}

// scene_view over the caller's arrays (src/renderer/scene_view.h:31-42), no copy.
scene_view view_of(const pt_scene_desc *d) {
    scene_view v{reinterpret_cast<const flat_triangle *>(d->triangles), reinterpret_cast<const flat_sphere *>(d->spheres),
                 reinterpret_cast<const flat_node *>(d->nodes), reinterpret_cast<const flat_material *>(d->materials),
                 reinterpret_cast<const flat_texture *>(d->textures), d->pixels, d->root, int32_t(d->node_count)};
    return v;
}

template <class F> void shard(size_t count, int threads, F fn) {
    if(threads < 1) threads = 1;
    if(size_t(threads) > count) threads = count ? int(count) : 1;
    std::vector<std::thread> pool;
    for(int t = 0; t < threads; t++) {
        size_t b = count*size_t(t)/size_t(threads), e = count*size_t(t+1)/size_t(threads);
        pool.emplace_back([=]() { fn(b, e, t); });
    }
    for(auto& th : pool) th.join();
}
} // namespace

struct ref_flat {
    flat_scene scene;
    flat_camera camera{};
    int has_camera = 0;
};

extern "C" {

int ref_validate(const pt_scene_desc *d) {
    try { validate_flat_scene(to_scene(d)); return 0; } catch(const std::exception&) { return 1; }
}

int ref_scene_lights(const pt_scene_desc *d, pt_light *out, size_t capacity, size_t *count, float *area) {
    try {
        auto scene = to_scene(d);
        auto lights = scene_lights(scene);
        *count = lights.size();
        for(size_t i = 0; i < lights.size() && i < capacity; i++) std::memcpy(&out[i], &lights[i], sizeof(pt_light));
        *area = lights.empty() ? 0 : lights.back().cumulative_area;
        return 0;
    } catch(const std::exception&) { return 1; }
}

// trace_world(host_view(scene), ray, tmin, tmax[i] or FLT_MAX, …) per ray, sharded over threads.
int ref_trace_world_batch(const pt_scene_desc *d, const pt_ray *rays, size_t count, float tmin,
                          const float *tmax, int brute, pt_trace_result *out, pt_ray_stats *stats, int threads) {
    scene_view view = view_of(d);
    auto r = reinterpret_cast<const ray *>(rays);
    shard(count, threads, [&](size_t b, size_t e, int) {
        for(size_t i = b; i < e; i++) {
            trace_result result{};
            trace_stats st;
            int error = 0;
            result.hit = trace_world(view, r[i], tmin, tmax ? tmax[i] : FLT_MAX, result.rec, brute != 0, error, st);
            result.error = error;
            std::memcpy(&out[i], &result, sizeof(result));
            if(stats) { stats[i].boxes = uint32_t(st.boxes); stats[i].primitives = uint32_t(st.primitives); }
        }
    });
    return 0;
}

// portable_renderer::add_samples's per-pixel loop (tests/support/portable_renderer.h:24-36),
// sharded over pixels.  sums/rng are in/out (reset them with ref_reset_pixels first).
int ref_render(const pt_scene_desc *d, const pt_camera *camera, int width, int height, int samples,
               int brute, int debug, int direct_light, float *sums, uint64_t *rng, uint64_t *rays, int threads) {
    try {
        auto scene = to_scene(d);
        validate_flat_scene(scene);
        auto lights = scene_lights(scene);
        scene_view view = host_view(scene, lights);
        flat_camera cam;
        std::memcpy(&cam, camera, sizeof cam);
        std::atomic<uint64_t> total{0};
        std::atomic<int> failed{0};
        size_t count = size_t(width)*size_t(height);
        shard(count, threads, [&](size_t b, size_t e, int) {
            uint64_t local = 0;
            for(size_t i = b; i < e; i++) {
                int x = int(i % size_t(width)), y = int(i / size_t(width));
                pixel_rng random;
                std::memcpy(&random, &rng[2*i], sizeof random);
                vec3 acc(sums[3*i], sums[3*i+1], sums[3*i+2]);
                int error = 0;
                for(int s = 0; s < samples; s++)
                    acc += trace_pixel_sample(view, cam, x, y, width, height, random, brute != 0,
                                              render_debug(debug), error, direct_light != 0, &local);
                if(error) failed = 1;
                sums[3*i] = acc.x(); sums[3*i+1] = acc.y(); sums[3*i+2] = acc.z();
                std::memcpy(&rng[2*i], &random, sizeof random);
            }
            total += local;
        });
        *rays += total.load();
        return failed.load() ? 2 : 0;
    } catch(const std::exception&) { return 1; }
}

void ref_reset_pixels(int width, int height, uint64_t seed, float *sums, uint64_t *rng) {
    size_t count = size_t(width)*size_t(height);
    for(size_t i = 0; i < count; i++) {
        pixel_rng r; r.seed(seed, i);
        sums[3*i] = sums[3*i+1] = sums[3*i+2] = 0;
        std::memcpy(&rng[2*i], &r, sizeof r);
    }
}

// The reference's own portable_renderer, single thread: image() means and ray count.
int ref_portable_image(const pt_scene_desc *d, const pt_camera *camera, int width, int height, uint64_t seed,
                       int brute, int debug, int direct_light, const int *batches, int batch_count,
                       float *image, uint64_t *rays) {
    try {
        auto scene = to_scene(d);
        flat_camera cam;
        std::memcpy(&cam, camera, sizeof cam);
        portable_renderer renderer(scene, cam, width, height, seed, brute != 0, render_debug(debug), direct_light != 0);
        for(int b = 0; b < batch_count; b++) renderer.add_samples(batches[b]);
        auto pixels = renderer.image();
        for(size_t i = 0; i < pixels.size(); i++) { image[3*i] = pixels[i].x(); image[3*i+1] = pixels[i].y(); image[3*i+2] = pixels[i].z(); }
        *rays = renderer.rays_traced();
        return 0;
    } catch(const std::exception&) { return 1; }
}

// display_pixels(image) (src/display/display_pixels.h:11-21)
void ref_display_pixels(const float *rgb, size_t pixels, unsigned char *rgba) {
    std::vector<vec3> linear(pixels);
    for(size_t i = 0; i < pixels; i++) linear[i] = vec3(rgb[3*i], rgb[3*i+1], rgb[3*i+2]);
    auto bytes = display_pixels(linear);
    std::memcpy(rgba, bytes.data(), bytes.size());
}

// pixel_rng stream draws (src/renderer/random.h)
void ref_rng_draws(uint64_t seed, uint64_t pixel, int count, float *uniforms, uint32_t *raw) {
    pixel_rng a, b; a.seed(seed, pixel); b.seed(seed, pixel);
    for(int i = 0; i < count; i++) { uniforms[i] = a.uniform(); raw[i] = b.next(); }
}

// flat primitive tests (src/flat/flat_intersect.h) and trace_box (src/renderer/transport.h:14-31)
int ref_triangle_hit(const pt_triangle *t, const pt_ray *r, float tmin, float tmax, pt_flat_hit *out) {
    flat_hit rec{};
    bool hit = flat_triangle_hit(*reinterpret_cast<const flat_triangle *>(t), *reinterpret_cast<const ray *>(r), tmin, tmax, rec);
    if(hit) std::memcpy(out, &rec, sizeof rec);
    return hit;
}
int ref_sphere_hit(const pt_sphere *s, const pt_ray *r, float tmin, float tmax, pt_flat_hit *out) {
    flat_hit rec{};
    bool hit = flat_sphere_hit(*reinterpret_cast<const flat_sphere *>(s), *reinterpret_cast<const ray *>(r), tmin, tmax, rec);
    if(hit) std::memcpy(out, &rec, sizeof rec);
    return hit;
}
int ref_trace_box(const pt_node *n, const pt_ray *r, float low, float high) {
    return trace_box(*reinterpret_cast<const flat_node *>(n), *reinterpret_cast<const ray *>(r), low, high);
}

// ---- reference scene construction: bvh_node (drand48 after srand48(seed)) + flatten_scene ----
ref_flat *ref_flat_from_desc(const pt_scene_desc *d) {
    auto h = new ref_flat;
    h->scene = to_scene(d);
    return h;
}

// triangle_mesh over the given faces (one material per face, constant-texture lambertian or
// diffuse_light), flattened as the reference exports it.  kinds: 0 lambertian, 3 light.
ref_flat *ref_flat_mesh(const pt_vec3 *vertices, const pt_vec3 *colors, const int *kinds, int faces, long seed) {
    try {
        srand48(seed);
        static std::vector<std::unique_ptr<texture>> textures;
        static std::vector<std::unique_ptr<material>> materials;
        std::vector<triangle> list;
        for(int f = 0; f < faces; f++) {
            textures.emplace_back(new constant_texture(vec3(colors[f].x, colors[f].y, colors[f].z)));
            if(kinds[f] == FLAT_LIGHT) materials.emplace_back(new diffuse_light(textures.back().get()));
            else materials.emplace_back(new lambertian(textures.back().get()));
            auto v = [&](int k) { return vec3(vertices[3*f+k].x, vertices[3*f+k].y, vertices[3*f+k].z); };
            list.emplace_back(v(0), v(1), v(2), materials.back().get());
        }
        triangle_mesh mesh(std::move(list));
        auto h = new ref_flat;
        h->scene = flatten_scene(&mesh);
        return h;
    } catch(const std::exception&) { return nullptr; }
}

// The CLI's scene pipeline (src/app/main.cpp:27-32): srand48(seed), obj_scene, flatten_scene,
// camera(lookfrom, lookat, (0,1,0), 40, aspect, 0, focus, 0, 1).
ref_flat *ref_flat_obj(const char *path, int width, int height, const float *scale, const float *rotate,
                       const float *translate, long seed, char *error, size_t capacity) {
    try {
        srand48(seed);
        float aspect = float(width)/height;
        obj_scene source(path, aspect, mesh_transform(vec3(scale[0],scale[1],scale[2]), vec3(rotate[0],rotate[1],rotate[2]),
                                                      vec3(translate[0],translate[1],translate[2])));
        auto h = new ref_flat;
        h->scene = flatten_scene(&source);
        camera cam(source.lookfrom, source.lookat, vec3(0,1,0), 40, aspect, 0, source.focus_dist, 0, 1);
        h->camera = flatten_camera(cam);
        h->has_camera = 1;
        return h;
    } catch(const std::exception& e) {
        if(error && capacity) { std::strncpy(error, e.what(), capacity-1); error[capacity-1] = 0; }
        return nullptr;
    }
}

// The reference camera (src/core/camera.h:16-43) flattened.
void ref_camera(const float *lookfrom, const float *lookat, const float *vup, float vfov, float aspect,
                float aperture, float focus, float t0, float t1, pt_camera *out) {
    camera c(vec3(lookfrom[0],lookfrom[1],lookfrom[2]), vec3(lookat[0],lookat[1],lookat[2]), vec3(vup[0],vup[1],vup[2]),
             vfov, aspect, aperture, focus, t0, t1);
    flat_camera f = flatten_camera(c);
    std::memcpy(out, &f, sizeof f);
}

void ref_flat_counts(const ref_flat *h, size_t *counts, int32_t *root, int32_t *max_depth) {
    counts[0] = h->scene.triangles.size(); counts[1] = h->scene.spheres.size(); counts[2] = h->scene.nodes.size();
    counts[3] = h->scene.materials.size(); counts[4] = h->scene.textures.size(); counts[5] = h->scene.pixels.size();
    *root = h->scene.root; *max_depth = h->scene.max_depth;
}
void ref_flat_copy(const ref_flat *h, pt_triangle *t, pt_sphere *s, pt_node *n, pt_material *m, pt_texture *x,
                   unsigned char *p, pt_camera *camera) {
    auto cp = [](void *dst, const void *src, size_t bytes) { if(bytes) std::memcpy(dst, src, bytes); };
    cp(t, h->scene.triangles.data(), h->scene.triangles.size()*sizeof(flat_triangle));
    cp(s, h->scene.spheres.data(), h->scene.spheres.size()*sizeof(flat_sphere));
    cp(n, h->scene.nodes.data(), h->scene.nodes.size()*sizeof(flat_node));
    cp(m, h->scene.materials.data(), h->scene.materials.size()*sizeof(flat_material));
    cp(x, h->scene.textures.data(), h->scene.textures.size()*sizeof(flat_texture));
    cp(p, h->scene.pixels.data(), h->scene.pixels.size());
    if(camera && h->has_camera) std::memcpy(camera, &h->camera, sizeof(flat_camera));
}
void ref_flat_free(ref_flat *h) { delete h; }

// ---- the pre-CUDA host path: triangle objects under the reference bvh_node, virtual hit() ----
struct ref_mesh { std::unique_ptr<triangle_mesh> mesh; };
ref_mesh *ref_mesh_create(const pt_vec3 *vertices, size_t faces, long seed) {
    srand48(seed);
    std::vector<triangle> list;
    list.reserve(faces);
    for(size_t f = 0; f < faces; f++) {
        auto v = [&](int k) { return vec3(vertices[3*f+k].x, vertices[3*f+k].y, vertices[3*f+k].z); };
        list.emplace_back(v(0), v(1), v(2), nullptr);
    }
    auto h = new ref_mesh;
    h->mesh.reset(new triangle_mesh(std::move(list)));
    return h;
}
// mesh.hit(ray, tmin, FLT_MAX) per ray (tests/mesh_validation.cpp:76-81); t_out = t or -1.
void ref_mesh_hit(const ref_mesh *h, const pt_ray *rays, size_t count, float tmin, float *t_out, int threads) {
    auto r = reinterpret_cast<const ray *>(rays);
    shard(count, threads, [&](size_t b, size_t e, int) {
        for(size_t i = b; i < e; i++) {
            hit_record rec;
            t_out[i] = h->mesh->hit(r[i], tmin, MAXFLOAT, rec) ? rec.t : -1.0f;
        }
    });
}
void ref_mesh_free(ref_mesh *h) { delete h; }

} // extern "C"
