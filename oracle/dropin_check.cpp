// dropin_check.cpp — the reference's own scene code driving the new library (TEST INFRASTRUCTURE ONLY).
//
// Built by oracle/Makefile against the reference's headers and its src/cuda/cuda_renderer.cu
// (where they lie) plus libptb200.so, into oracle/_ref/dropin_check.  It builds a scene with
// the reference's classes (sphere, bvh_node, materials, camera, flatten_scene), then renders and
// queries it twice through the same calls: once with the reference's cuda_renderer /
// cuda_query_rays, once with ptb::cuda_renderer / ptb::cuda_query_rays from
// include/pt_cuda_renderer.hpp — the reference's own flat_scene, flat_camera, ray, trace_result
// and vec3 types pass unchanged.  Exit 0 when images, ray counts and query records agree
// bit for bit, 1 otherwise, 77 without a device (the reference's skip code).
#include <cstdio>
#include <cstring>
#include <random>
#include "cuda/cuda_renderer.h"
#include "flat/flat_export.h"
#include "../include/pt_cuda_renderer.hpp"

int main() {
    std::string device;
    if(!cuda_device_available(device)) { std::printf("SKIP: %s\n", device.c_str()); return 77; }
    constant_texture paint(vec3(0.3, 0.7, 0.2)), lamp_color(vec3(4, 3, 2));
    lambertian diffuse(&paint);
    metal mirror(vec3(0.8, 0.7, 0.6), 0.1);
    dielectric glass(1.5);
    diffuse_light lamp(&lamp_color);
    sphere a(vec3(-2, 0, 0), 1, &diffuse), b(vec3(0, 0, 0), 1, &glass), c(vec3(2, 0, 0), 1, &mirror);
    sphere ground(vec3(0, -101, 0), 100, &diffuse), light(vec3(0, 4, 2), 2, &lamp);
    hitable *objects[] = {&a, &b, &c, &ground, &light};
    srand48(19);
    bvh_node world(objects, 5, 0, 1);
    flat_scene flat = flatten_scene(&world);
    camera view(vec3(0, 2, 8), vec3(0, 0, 0), vec3(0, 1, 0), 40, 1.5, 0.2, 8, 0.2, 0.8);
    flat_camera fc = flatten_camera(view);
    int failures = 0;
    for(int debug = DEBUG_SHADED; debug <= DEBUG_INTERSECTIONS; debug++) {
        for(bool mis : {true, false}) {
            cuda_renderer ref(flat, fc, 31, 21, 19, false, render_debug(debug), mis);
            ptb::basic_cuda_renderer<vec3> ours(flat, fc, 31, 21, 19, false, debug, mis);
            ref.add_samples(16); ref.add_samples(48);
            ours.add_samples(16); ours.add_samples(48);
            auto x = ref.image(), y = ours.image();
            bool same = x.size() == y.size() && std::memcmp(x.data(), y.data(), x.size() * sizeof(vec3)) == 0 &&
                        ref.rays_traced() == ours.rays_traced() && ref.sample_count() == ours.sample_count() &&
                        ref.rgba_image() == ours.rgba_image();
            std::printf("render debug=%d mis=%d rays=%llu/%llu %s\n", debug, int(mis), (unsigned long long)ref.rays_traced(),
                        (unsigned long long)ours.rays_traced(), same ? "identical" : "DIFFERENT");
            failures += !same;
        }
    }
    std::vector<ray> rays;
    std::mt19937 rng(7);
    for(int i = 0; i < 4096; i++) {
        float u = float(double(rng()) / 4294967296.0), v = float(double(rng()) / 4294967296.0);
        rays.push_back(view.get_ray(u, v));
    }
    for(bool brute : {false, true}) {
        auto x = cuda_query_rays(flat, rays, brute);
        auto y = ptb::cuda_query_rays<trace_result>(flat, rays, brute);
        bool same = x.size() == y.size();
        for(size_t i = 0; same && i < x.size(); i++) {
            // sphere UVs come from atan2f/asinf on both sides: same device functions, same bits
            same = std::memcmp(&x[i], &y[i], sizeof(trace_result)) == 0;
        }
        std::printf("query brute=%d %s\n", int(brute), same ? "identical" : "DIFFERENT");
        failures += !same;
    }
    bool rejected = false;
    try { ptb::cuda_renderer bad(flat, fc, 0, 21, 19); } catch(const std::invalid_argument &) { rejected = true; }
    std::printf("invalid dimensions rejected: %s\n", rejected ? "yes" : "NO");
    failures += !rejected;
    return failures ? 1 : 0;
}
