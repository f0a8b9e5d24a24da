// ray_tracer — the reference's command-line renderer (src/app/main.cpp:9-52) on this library.
//
// Same flags, defaults, validation messages, exit codes (0; 1 on an error, after printing it and
// "Use --help for usage."; 77 without a CUDA device) and output: an ASCII PPM (P3) of the
// gamma-2 image on stdout, rows from the top, device / scene / render notes on stderr.
// The scene is the OBJ with the reference's preview stage (pt_workload_obj); the render is
// pt_renderer with the reference's bounce limit (50), MIS unless --lighting classic.
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>
#include "pt.h"
#include "pt_workloads.h"

namespace {

struct Options {
    int width = 500, height = 500, samples = 100, seed = 7, batch_samples = 16;
    int debug = PT_DEBUG_SHADED;
    std::string obj_file;
    std::string backend = "cuda";
    float scale[3] = {1, 1, 1}, rotate[3] = {0, 0, 0}, translate[3] = {0, 0, 0};
    bool help = false, direct_light = true;
};

std::string default_obj() {
    const char *dir = std::getenv("RAY_TRACER_ASSET_DIR");
    return std::string(dir && *dir ? dir : "assets") + "/models/blender_sphere/sphere.obj";
}

// parse_integer / parse_float (src/app/render_options.h:29-47)
int parse_integer(const char *value, int minimum) {
    char *end;
    errno = 0;
    long parsed = std::strtol(value, &end, 10);
    if (errno || end == value || *end != '\0' || parsed < minimum || parsed > INT_MAX)
        throw std::invalid_argument(std::string("invalid integer: ") + value);
    return int(parsed);
}

float parse_float(const char *value) {
    char *end;
    errno = 0;
    float parsed = std::strtof(value, &end);
    if (errno || end == value || *end != '\0' || !std::isfinite(parsed))
        throw std::invalid_argument(std::string("invalid finite number: ") + value);
    return parsed;
}

// parse_options (src/app/render_options.h:49-107)
Options parse_options(int argc, char **argv) {
    Options o;
    o.obj_file = default_obj();
    bool has_transform = false, has_obj = false;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        if (a == "--help") {
            o.help = true;
        } else if (a == "--lighting") {
            if (i + 1 >= argc) throw std::invalid_argument("missing value for --lighting");
            std::string v = argv[++i];
            if (v != "classic" && v != "mis") throw std::invalid_argument("lighting must be classic or mis");
            o.direct_light = v == "mis";
        } else if (a == "--normals") {
            o.debug = PT_DEBUG_NORMALS;
        } else if (a == "--obj-scale" || a == "--obj-rotate" || a == "--obj-translate") {
            if (i + 3 >= argc) throw std::invalid_argument("expected three values for " + a);
            float *dst = a == "--obj-scale" ? o.scale : a == "--obj-rotate" ? o.rotate : o.translate;
            for (int k = 0; k < 3; k++) dst[k] = parse_float(argv[++i]);
            has_transform = true;
        } else if (a == "--width" || a == "--height" || a == "--samples" || a == "--seed" || a == "--obj" || a == "--backend" ||
                   a == "--debug" || a == "--batch-samples") {
            if (i + 1 >= argc) throw std::invalid_argument("missing value for " + a);
            const char *v = argv[++i];
            if (a == "--obj") { o.obj_file = v; has_obj = true; }
            else if (a == "--backend") o.backend = v;
            else if (a == "--debug") {
                std::string m = v;
                if (m == "shaded") o.debug = PT_DEBUG_SHADED;
                else if (m == "normals") o.debug = PT_DEBUG_NORMALS;
                else if (m == "triangle-id") o.debug = PT_DEBUG_TRIANGLE;
                else if (m == "material-id") o.debug = PT_DEBUG_MATERIAL;
                else if (m == "bvh") o.debug = PT_DEBUG_BVH;
                else if (m == "intersections") o.debug = PT_DEBUG_INTERSECTIONS;
                else throw std::invalid_argument("unknown debug mode: " + m);
            } else if (a == "--batch-samples") o.batch_samples = parse_integer(v, 1);
            else if (a == "--width") o.width = parse_integer(v, 1);
            else if (a == "--height") o.height = parse_integer(v, 1);
            else if (a == "--samples") o.samples = parse_integer(v, 1);
            else o.seed = parse_integer(v, 0);
        } else {
            throw std::invalid_argument("unknown option: " + a);
        }
    }
    if (o.obj_file.empty()) throw std::invalid_argument("OBJ filename must not be empty");
    if (has_transform && !has_obj) throw std::invalid_argument("OBJ transforms require --obj FILE");
    for (int k = 0; k < 3; k++)
        if (!std::isfinite(o.scale[k]) || o.scale[k] == 0 || !std::isfinite(o.rotate[k]) || !std::isfinite(o.translate[k]))
            throw std::invalid_argument("mesh transform requires finite values and nonzero scale");
    if (o.backend != "cuda") throw std::invalid_argument("CUDA is the only rendering backend");
    return o;
}

// color_channel (src/display/color.h:6-11)
int color_channel(float linear) {
    if (!(linear > 0)) return 0;
    if (linear >= 1) return 255;
    float gamma = std::sqrt(linear);
    return int(255.99 * gamma);
}

void check(pt_status st) {
    if (st == PT_OK) return;
    std::string message = pt_last_error();
    if (st == PT_INVALID_ARGUMENT) throw std::invalid_argument(message);
    throw std::runtime_error(message);
}

struct Handles {
    pt_flat *flat = nullptr;
    pt_scene *scene = nullptr;
    pt_renderer *renderer = nullptr;
    ~Handles() {
        if (renderer) pt_renderer_destroy(renderer);
        if (scene) pt_scene_destroy(scene);
        if (flat) pt_flat_destroy(flat);
    }
};

} // namespace

int main(int argc, char **argv) {
    try {
        Options o = parse_options(argc, argv);
        if (o.help) {
            std::cout << "Usage: ray_tracer [--obj FILE] [--width N] [--height N]\n"
                      << "  [--samples N] [--batch-samples N] [--seed N]\n"
                      << "  [--obj-scale X Y Z] [--obj-rotate X Y Z] [--obj-translate X Y Z]\n"
                      << "  [--debug shaded|normals|triangle-id|material-id|bvh|intersections] [--normals]\n"
                      << "  [--lighting classic|mis] (default: mis)\n"
                      << "Defaults: CUDA, Blender sphere ($RAY_TRACER_ASSET_DIR/models/blender_sphere/sphere.obj), "
                      << "500x500, 100 samples/pixel, seed 7.\n"
                      << "PPM output goes to stdout. OBJ transforms apply scale, XYZ rotation in degrees, then translation.\n";
            return 0;
        }
        char device[256];
        if (!pt_device_available(device, sizeof device)) {
            std::cerr << "CUDA device unavailable: " << device << '\n';
            return 77;
        }
        Handles h;
        pt_camera camera;
        std::vector<char> warnings(1 << 16);
        check(pt_workload_obj(o.obj_file.c_str(), o.width, o.height, o.scale, o.rotate, o.translate, &h.flat, &camera,
                              warnings.data(), warnings.size()));
        pt_scene_desc desc;
        check(pt_flat_desc(h.flat, &desc));
        check(pt_scene_create(&desc, &h.scene));
        check(pt_renderer_create(h.scene, &camera, o.width, o.height, uint64_t(o.seed), o.direct_light ? PT_RENDER_MIS : 0,
                                 o.debug, 50, &h.renderer));
        std::cerr << "CUDA: " << device << "\nLoaded " << desc.triangle_count << " triangles, " << desc.node_count
                  << " BVH nodes\n" << warnings.data();
        int count = 0;
        while (count < o.samples) {
            check(pt_add_samples(h.renderer, std::min(o.batch_samples, o.samples - count)));
            check(pt_stats(h.renderer, &count, nullptr, nullptr));
        }
        std::vector<float> pixels(size_t(o.width) * size_t(o.height) * 3);
        check(pt_get_image(h.renderer, pixels.data(), pixels.size()));
        std::cerr << "Rendered " << o.width << "x" << o.height << ", " << count << " samples/pixel\n";
        std::cout << "P3\n" << o.width << " " << o.height << "\n255\n";
        for (int y = o.height - 1; y >= 0; y--) {
            for (int x = 0; x < o.width; x++) {
                const float *p = &pixels[(size_t(y) * size_t(o.width) + size_t(x)) * 3];
                std::cout << color_channel(p[0]) << " " << color_channel(p[1]) << " " << color_channel(p[2]) << '\n';
            }
        }
        if (!std::cout) throw std::runtime_error("could not write image output");
    } catch (const std::exception &error) {
        std::cerr << error.what() << "\nUse --help for usage.\n";
        return 1;
    }
    return 0;
}
