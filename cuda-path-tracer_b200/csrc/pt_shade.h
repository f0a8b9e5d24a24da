// pt_shade.h — per-bounce shading of the MIS path tracer (device), same arithmetic as the
// reference's trace_color pieces so a path makes the same decisions and sums the same floats.
//
//   textures         src/renderer/transport.h:87-111
//   scatter          src/renderer/transport.h:113-155
//   light sampling   src/renderer/light_sampling.h:10-73
//   emitter lookup   binary search over the cumulative-area table (scene_lights)
#pragma once

#include <cmath>
#include "pt_traverse.h"

namespace ptb {

// trace_image: nearest texel, V flipped, clamped (transport.h:87-101)
__device__ inline f3 trace_image(const DeviceScene &scene, const pt_texture &tex, float u, float v) {
    u = fminf(1.0f, fmaxf(0.0f, u));
    v = fminf(1.0f, fmaxf(0.0f, v));
    int i = u * tex.width;
    int j = (1 - v) * tex.height - 0.001;
    if (i < 0) i = 0;
    if (j < 0) j = 0;
    if (i > tex.width - 1) i = tex.width - 1;
    if (j > tex.height - 1) j = tex.height - 1;
    size_t offset = size_t(tex.byte_offset) + 3 * size_t(i) + 3 * size_t(tex.width) * size_t(j);
    float red = int(scene.pixels[offset]) / 255.0;
    float green = int(scene.pixels[offset + 1]) / 255.0;
    float blue = int(scene.pixels[offset + 2]) / 255.0;
    return mk(red, green, blue);
}

__device__ inline f3 trace_texture(const DeviceScene &scene, int32_t id, float u, float v) {
    const pt_texture &tex = scene.textures[id];
    if (tex.type == PT_TEX_CONSTANT) return mk(tex.color);
    if (tex.type == PT_TEX_IMAGE) return trace_image(scene, tex, u, v);
    u = u * tex.scale.x + tex.offset.x;
    v = v * tex.scale.y + tex.offset.y;
    if (!tex.clamp) { u -= floor(u); v -= floor(v); }
    return mk(tex.color) * trace_image(scene, scene.textures[tex.image_id], u, v);
}

__device__ inline f3 trace_reflect(f3 v, f3 n) { return v - 2 * dot(v, n) * n; }

// mis_weight: power heuristic, scaled before squaring (light_sampling.h:10-16)
__device__ inline float mis_weight(float a, float b) {
    float scale = fmaxf(a, b);
    if (!(scale > 0)) return 0;
    a /= scale; b /= scale;
    return a * a / (a * a + b * b);
}

// cosine_direction (light_sampling.h:18-25)
__device__ inline f3 cosine_direction(f3 normal, Pcg &random) {
    float u = random.uniform(), v = random.uniform();
    float radius = sqrtf(u), angle = 2 * float(M_PI) * v;
    f3 helper = fabsf(normal.x) > 0.9f ? mk(0, 1, 0) : mk(1, 0, 0);
    f3 tangent = unit(cross(helper, normal));
    f3 bitangent = cross(normal, tangent);
    return radius * cosf(angle) * tangent + radius * sinf(angle) * bitangent + sqrtf(1 - u) * normal;
}

struct LightSample { f3 point, normal; float u, v; int material; };

// sample_light: area-weighted emitter choice, uniform point on it (light_sampling.h:27-54)
__device__ inline LightSample sample_light(const DeviceScene &scene, Pcg &random) {
    float choice = random.uniform() * scene.light_area;
    int low = 0, high = scene.light_count - 1;
    while (low < high) {
        int middle = low + (high - low) / 2;
        if (choice < scene.lights[middle].cumulative_area) high = middle;
        else low = middle + 1;
    }
    const pt_light &light = scene.lights[low];
    float u = random.uniform(), v = random.uniform();
    LightSample result;
    if (light.type == PT_TRIANGLE) {
        const pt_triangle &t = scene.triangles[light.primitive];
        float root = sqrtf(u), a = 1 - root, b = root * (1 - v), c = root * v;
        result.point = a * mk(t.v0) + b * mk(t.v1) + c * mk(t.v2);
        result.normal = unit(cross(mk(t.v1) - mk(t.v0), mk(t.v2) - mk(t.v0)));
        f3 uv = a * mk(t.uv0) + b * mk(t.uv1) + c * mk(t.uv2);
        result.u = uv.x; result.v = uv.y; result.material = t.material_id;
    } else {
        const pt_sphere &s = scene.sphere_src[light.primitive];
        float z = 1 - 2 * u, radius = sqrtf(fmaxf(0, 1 - z * z)), angle = 2 * float(M_PI) * v;
        result.normal = mk(radius * cosf(angle), z, radius * sinf(angle));
        result.point = mk(s.center) + fabsf(s.radius) * result.normal;
        if (s.radius < 0) result.normal = -result.normal;
        sphere_uv(result.normal, result.u, result.v);
        result.material = s.material_id;
    }
    return result;
}

// light_direction_pdf (light_sampling.h:56-65)
__device__ inline float light_direction_pdf(float area, f3 from, f3 point, f3 normal) {
    f3 delta = point - from;
    float distance_squared = sqlen(delta);
    if (!(area > 0) || !(distance_squared > 0)) return 0;
    float cosine = fabsf(dot(normal, delta)) / sqrtf(distance_squared);
    if (!(cosine > 0)) return 0;
    float pdf = distance_squared / (cosine * area);
    return finite(pdf) ? pdf : 0;
}

// hit_light_pdf (light_sampling.h:67-73)
__device__ inline float hit_light_pdf(const DeviceScene &scene, f3 from, const pt_flat_hit &hit) {
    f3 normal = mk(hit.normal);
    if (hit.primitive_type == PT_TRIANGLE) {
        const pt_triangle &t = scene.triangles[hit.primitive_id];
        normal = unit(cross(mk(t.v1) - mk(t.v0), mk(t.v2) - mk(t.v0)));
    }
    return light_direction_pdf(scene.light_area, from, mk(hit.p), normal);
}

// trace_scatter (transport.h:115-155)
__device__ inline bool trace_scatter(const DeviceScene &scene, const pt_material &mat, f3 in_dir,
                                     const pt_flat_hit &rec, Pcg &random, f3 &attenuation, f3 &out_dir) {
    f3 p = mk(rec.p), n = mk(rec.normal);
    if (mat.type == PT_DIFFUSE) {
        f3 target = p + n + sample_ball(random);
        out_dir = target - p;
        attenuation = trace_texture(scene, mat.texture_id, rec.u, rec.v);
        return true;
    }
    if (mat.type == PT_METAL) {
        f3 reflected = trace_reflect(unit(in_dir), n);
        f3 ball = sample_ball(random);
        out_dir = reflected + mat.fuzz * ball;
        attenuation = mk(mat.albedo);
        return dot(out_dir, n) > 0;
    }
    if (mat.type == PT_GLASS) {
        f3 outward, refracted = mk(0, 0, 0);
        f3 reflected = trace_reflect(in_dir, n);
        float ratio, cosine;
        if (dot(in_dir, n) > 0) {
            outward = -n; ratio = mat.ref_idx;
            cosine = mat.ref_idx * dot(in_dir, n) / length(in_dir);
        } else {
            outward = n; ratio = 1.0f / mat.ref_idx;
            cosine = -dot(in_dir, n) / length(in_dir);
        }
        f3 uv = unit(in_dir);
        float dt = dot(uv, outward);
        float discriminant = 1.0f - ratio * ratio * (1 - dt * dt);
        float probability = 1;
        if (discriminant > 0) {
            refracted = ratio * (uv - outward * dt) - outward * sqrt(discriminant);
            float r0 = (1 - mat.ref_idx) / (1 + mat.ref_idx);
            r0 *= r0;
            probability = r0 + (1 - r0) * pow(1 - cosine, 5);
        }
        if (random.uniform() < probability) out_dir = reflected;
        else out_dir = refracted;
        attenuation = mk(1, 1, 1);
        return true;
    }
    return false;
}

// id_color (transport.h:164-167)
__device__ inline f3 id_color(int id) {
    uint32_t bits = (uint32_t(id) + 1u) * 2654435761u;
    return mk((bits & 255) / 255.0f, ((bits >> 8) & 255) / 255.0f, ((bits >> 16) & 255) / 255.0f);
}

} // namespace ptb
