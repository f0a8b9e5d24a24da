// ref_cuda_shim.cu — C entry points around the reference's OWN CUDA renderer (TEST INFRASTRUCTURE ONLY).
//
// oracle/Makefile compiles this file together with the reference's src/cuda/cuda_renderer.cu,
// where it lies, for sm_100a with --fmad=false (the reference's own flag, CMakeLists.txt:19-20)
// into oracle/_ref/libref_cuda.so.  It lets GPU tests compare the new kernels with the
// reference's kernels on the same B200 and lets the benches time them.  No restatement: every
// call goes to class cuda_renderer / cuda_query_rays (src/cuda/cuda_renderer.h:8-32).
#include <cstring>
#include <memory>
#include "cuda/cuda_renderer.h"
#include "../include/pt.h"

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
thread_local std::string last_error;
}

extern "C" {

const char *refgpu_last_error() { return last_error.c_str(); }

int refgpu_available(char *buf, size_t capacity) {
    std::string description;
    bool ok = cuda_device_available(description);
    if(buf && capacity) { std::strncpy(buf, description.c_str(), capacity-1); buf[capacity-1] = 0; }
    return ok ? 1 : 0;
}

int refgpu_query(const pt_scene_desc *d, const pt_ray *rays, size_t count, int brute, pt_trace_result *out) {
    try {
        std::vector<ray> list(count);
        if(count) std::memcpy(list.data(), rays, count*sizeof(ray));
        auto results = cuda_query_rays(to_scene(d), list, brute != 0);
        if(count) std::memcpy(out, results.data(), count*sizeof(trace_result));
        return 0;
    } catch(const std::exception& e) { last_error = e.what(); return 1; }
}

void *refgpu_renderer_create(const pt_scene_desc *d, const pt_camera *camera, int width, int height, uint64_t seed,
                             int brute, int debug, int direct_light) {
    try {
        flat_camera cam;
        std::memcpy(&cam, camera, sizeof cam);
        return new cuda_renderer(to_scene(d), cam, width, height, seed, brute != 0, render_debug(debug), direct_light != 0);
    } catch(const std::exception& e) { last_error = e.what(); return nullptr; }
}
int refgpu_add_samples(void *h, int count) {
    try { static_cast<cuda_renderer *>(h)->add_samples(count); return 0; }
    catch(const std::exception& e) { last_error = e.what(); return 1; }
}
int refgpu_set_block_shape(void *h, int w, int hh) {
    try { static_cast<cuda_renderer *>(h)->set_block_shape(w, hh); return 0; }
    catch(const std::exception& e) { last_error = e.what(); return 1; }
}
int refgpu_reset(void *h, const pt_camera *camera) {
    try {
        flat_camera cam; std::memcpy(&cam, camera, sizeof cam);
        static_cast<cuda_renderer *>(h)->reset(cam); return 0;
    } catch(const std::exception& e) { last_error = e.what(); return 1; }
}
int refgpu_image(void *h, float *rgb) {
    try {
        auto img = static_cast<cuda_renderer *>(h)->image();
        for(size_t i = 0; i < img.size(); i++) { rgb[3*i] = img[i].x(); rgb[3*i+1] = img[i].y(); rgb[3*i+2] = img[i].z(); }
        return 0;
    } catch(const std::exception& e) { last_error = e.what(); return 1; }
}
int refgpu_rgba(void *h, unsigned char *rgba) {
    try {
        auto bytes = static_cast<cuda_renderer *>(h)->rgba_image();
        std::memcpy(rgba, bytes.data(), bytes.size());
        return 0;
    } catch(const std::exception& e) { last_error = e.what(); return 1; }
}
void refgpu_stats(void *h, int *samples, float *ms, uint64_t *rays) {
    auto r = static_cast<cuda_renderer *>(h);
    *samples = r->sample_count(); *ms = r->kernel_milliseconds(); *rays = r->rays_traced();
}
void refgpu_destroy(void *h) { delete static_cast<cuda_renderer *>(h); }

} // extern "C"
