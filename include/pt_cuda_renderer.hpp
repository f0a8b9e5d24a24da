// pt_cuda_renderer.hpp — C++17 drop-in for the reference's renderer surface, over the C ABI.
//
// Replaces src/cuda/cuda_renderer.h:8-32 of AdmiralHeathCL/cuda-path-tracer:
//   bool cuda_device_available(std::string&);
//   class cuda_renderer { ctor(scene, camera, w, h, seed, brute, debug, direct_light); reset;
//                         add_samples; set_block_shape; image; rgba_image; write_rgba;
//                         sample_count; kernel_milliseconds; rays_traced };
//   std::vector<trace_result> cuda_query_rays(const flat_scene&, const std::vector<ray>&, bool);
// The templates accept the reference's own flat_scene / flat_camera / ray / trace_result / vec3
// types (or any types with the same members and byte layout), so a caller swaps
// `#include "cuda/cuda_renderer.h"` for this header and the `ptb::` names.  Errors throw the
// reference's exception types: std::invalid_argument for bad arguments, std::runtime_error for
// invalid scenes, CUDA failures and traversal stack overflow.
#pragma once

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>
#include "pt.h"

namespace ptb {

inline void throw_status(pt_status status) {
    if(status == PT_OK) return;
    std::string message = pt_last_error();
    if(status == PT_INVALID_ARGUMENT) throw std::invalid_argument(message);
    throw std::runtime_error(message);
}

inline bool cuda_device_available(std::string &description) {
    char buffer[256];
    int ok = pt_device_available(buffer, sizeof buffer);
    description = buffer;
    return ok != 0;
}

// pt_scene_desc over a flat_scene's vectors (no copy; the library copies on upload).
template <class FlatScene> pt_scene_desc scene_desc(const FlatScene &s) {
    static_assert(sizeof(*s.triangles.data()) == sizeof(pt_triangle), "flat_triangle layout");
    static_assert(sizeof(*s.spheres.data()) == sizeof(pt_sphere), "flat_sphere layout");
    static_assert(sizeof(*s.nodes.data()) == sizeof(pt_node), "flat_node layout");
    static_assert(sizeof(*s.materials.data()) == sizeof(pt_material), "flat_material layout");
    static_assert(sizeof(*s.textures.data()) == sizeof(pt_texture), "flat_texture layout");
    pt_scene_desc d{};
    d.triangles = reinterpret_cast<const pt_triangle *>(s.triangles.data()); d.triangle_count = s.triangles.size();
    d.spheres = reinterpret_cast<const pt_sphere *>(s.spheres.data()); d.sphere_count = s.spheres.size();
    d.nodes = reinterpret_cast<const pt_node *>(s.nodes.data()); d.node_count = s.nodes.size();
    d.materials = reinterpret_cast<const pt_material *>(s.materials.data()); d.material_count = s.materials.size();
    d.textures = reinterpret_cast<const pt_texture *>(s.textures.data()); d.texture_count = s.textures.size();
    d.pixels = reinterpret_cast<const unsigned char *>(s.pixels.data()); d.pixel_bytes = s.pixels.size();
    d.root = s.root; d.max_depth = s.max_depth;
    return d;
}

// Owning device scene.
class device_scene {
public:
    template <class FlatScene> explicit device_scene(const FlatScene &scene) {
        pt_scene_desc d = scene_desc(scene);
        throw_status(pt_scene_create(&d, &handle_));
    }
    ~device_scene() { if(handle_) pt_scene_destroy(handle_); }
    device_scene(const device_scene &) = delete;
    device_scene &operator=(const device_scene &) = delete;
    const pt_scene *get() const { return handle_; }
private:
    pt_scene *handle_ = nullptr;
};

// class cuda_renderer (src/cuda/cuda_renderer.h:10-29).  `max_depth` defaults to the
// reference's hard-coded 50 (src/renderer/transport.h:174).
template <class Vec3 = pt_vec3> class basic_cuda_renderer {
public:
    template <class FlatScene, class FlatCamera>
    basic_cuda_renderer(const FlatScene &scene, const FlatCamera &camera, int width, int height, uint64_t seed,
                        bool brute = false, int debug = PT_DEBUG_SHADED, bool direct_light = false, int max_depth = 50)
        : scene_(std::make_unique<device_scene>(scene)), width_(width), height_(height) {
        static_assert(sizeof(FlatCamera) == sizeof(pt_camera), "flat_camera layout");
        uint32_t flags = (direct_light ? PT_RENDER_MIS : 0u) | (brute ? PT_RENDER_BRUTE : 0u);
        throw_status(pt_renderer_create(scene_->get(), reinterpret_cast<const pt_camera *>(&camera), width, height, seed,
                                        flags, debug, max_depth, &handle_));
    }
    ~basic_cuda_renderer() { if(handle_) pt_renderer_destroy(handle_); }
    basic_cuda_renderer(const basic_cuda_renderer &) = delete;
    basic_cuda_renderer &operator=(const basic_cuda_renderer &) = delete;

    template <class FlatCamera> void reset(const FlatCamera &camera) {
        throw_status(pt_reset(handle_, reinterpret_cast<const pt_camera *>(&camera)));
    }
    void add_samples(int count) { throw_status(pt_add_samples(handle_, count)); }
    void set_block_shape(int width, int height) { throw_status(pt_set_block_shape(handle_, width, height)); }
    std::vector<Vec3> image() const {
        static_assert(sizeof(Vec3) == 3 * sizeof(float), "vec3 layout");
        std::vector<Vec3> out(size_t(width_) * size_t(height_));
        throw_status(pt_get_image(handle_, reinterpret_cast<float *>(out.data()), out.size() * 3));
        return out;
    }
    std::vector<unsigned char> rgba_image() const {
        std::vector<unsigned char> out(4 * size_t(width_) * size_t(height_));
        throw_status(pt_rgba_image(handle_, out.data(), out.size()));
        return out;
    }
    void write_rgba(unsigned char *device_pixels, size_t bytes) const { throw_status(pt_write_rgba(handle_, device_pixels, bytes)); }
    int sample_count() const { int s = 0; throw_status(pt_stats(handle_, &s, nullptr, nullptr)); return s; }
    float kernel_milliseconds() const { float ms = 0; throw_status(pt_stats(handle_, nullptr, &ms, nullptr)); return ms; }
    uint64_t rays_traced() const { uint64_t r = 0; throw_status(pt_stats(handle_, nullptr, nullptr, &r)); return r; }
    // Resumable state: linear sums and the per-pixel PCG states.
    std::vector<float> sums() const {
        std::vector<float> out(3 * size_t(width_) * size_t(height_));
        throw_status(pt_get_sums(handle_, out.data(), out.size()));
        return out;
    }
    std::vector<uint64_t> rng_states() const {
        std::vector<uint64_t> out(2 * size_t(width_) * size_t(height_));
        throw_status(pt_get_rng(handle_, out.data(), out.size()));
        return out;
    }
private:
    std::unique_ptr<device_scene> scene_;
    pt_renderer *handle_ = nullptr;
    int width_, height_;
};
using cuda_renderer = basic_cuda_renderer<>;

// cuda_query_rays(scene, rays, brute) (src/cuda/cuda_renderer.h:32): full trace_result records.
template <class TraceResult = pt_trace_result, class FlatScene, class Ray>
std::vector<TraceResult> cuda_query_rays(const FlatScene &scene, const std::vector<Ray> &rays, bool brute = false) {
    static_assert(sizeof(Ray) == sizeof(pt_ray) && sizeof(TraceResult) == sizeof(pt_trace_result), "record layout");
    device_scene uploaded(scene);
    std::vector<TraceResult> out(rays.size());
    if(rays.empty()) return out;
    throw_status(pt_query_rays_compat(uploaded.get(), reinterpret_cast<const pt_ray *>(rays.data()), rays.size(),
                                      brute ? 1 : 0, reinterpret_cast<pt_trace_result *>(out.data())));
    return out;
}

} // namespace ptb
