// pt_wavefront.h — path records and the per-bounce step shared by the wavefront renderers
// (pt_render.cu: one image; pt_batch.cu: many jobs in one launch).
#pragma once

#include "pt_shade.h"

namespace ptb {

struct alignas(16) PathState {
    float ox, oy, oz, time;
    float dx, dy, dz, prev_pdf;
    float tr, tg, tb; int32_t depth;
    float rr, rg, rb; int32_t samples_left;
};
struct alignas(16) PathHit { float t, u, v; int32_t slot; };
struct alignas(16) ShadowRay {
    float ox, oy, oz, tmax;
    float dx, dy, dz, time;
    float cr, cg, cb; int32_t pixel;
};
static_assert(sizeof(PathState) == 64 && sizeof(PathHit) == 16 && sizeof(ShadowRay) == 48, "path records");

// What shading needs to know about the image a path belongs to.
struct ShadeCtx {
    const pt_camera *camera;
    int width, height, max_depth, debug, mis;
};

__device__ inline unsigned lane_id() { return threadIdx.x & 31; }

// Warp-aggregated append: one atomicAdd per warp.
__device__ inline void push(bool take, int32_t value, int32_t *queue, int32_t *counter) {
    unsigned m = __ballot_sync(0xffffffffu, take);
    if (!m) return;
    int leader = __ffs(m) - 1;
    int base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (take) queue[base + __popc(m & ((1u << lane_id()) - 1u))] = value;
}

// trace_pixel_sample's camera step (src/renderer/transport.h:232-239) for pixel (x, y) of a
// width x height image; starts a fresh path.
__device__ inline void camera_path(const pt_camera &camera, int width, int height, int32_t pixel, Pcg &rng, PathState &s) {
    int x = pixel % width, y = pixel / width;
    float u = (x + rng.uniform()) / float(width);
    float v = (y + rng.uniform()) / float(height);
    pt_ray r;
    camera_ray(camera, u, v, rng, r);
    s.ox = r.origin.x; s.oy = r.origin.y; s.oz = r.origin.z; s.time = r.time;
    s.dx = r.direction.x; s.dy = r.direction.y; s.dz = r.direction.z; s.prev_pdf = 0;
    s.tr = 1; s.tg = 1; s.tb = 1; s.depth = 0;
    s.rr = 0; s.rg = 0; s.rb = 0;
}

__device__ inline pt_ray path_ray(const PathState &s) {
    pt_ray r;
    r.origin = pt_vec3{s.ox, s.oy, s.oz};
    r.direction = pt_vec3{s.dx, s.dy, s.dz};
    r.time = s.time;
    return r;
}

// The rest of one trace_color iteration for the path in `slot`, rendering `pixel` (its index
// inside its image) (transport.h:179-228), given its closest
// hit: emission with its MIS weight, next-event estimation (which may emit a shadow ray),
// cosine or material scatter; when the sample ends, its radiance is added to the pixel sum and
// the pixel's next camera ray starts.  Returns whether the path is still live.
__device__ inline bool shade_path(const DeviceScene &scene, const ShadeCtx &p, float *sum, int32_t pixel, int32_t slot,
                                  PathState &s, const PathHit &h, const uint2 &stats, Pcg &rng, ShadowRay &sr, bool &shadow) {
    shadow = false;
    f3 radiance = mk(s.rr, s.rg, s.rb);
    f3 throughput = mk(s.tr, s.tg, s.tb);
    bool finished = false;
    if (p.debug == PT_DEBUG_BVH || p.debug == PT_DEBUG_INTERSECTIONS) {
        float cost = log2f(1.0f + float(p.debug == PT_DEBUG_BVH ? stats.x : stats.y)) / 10.0f;
        cost = fminf(1, cost);
        radiance = mk(cost, cost * cost, 1 - cost);
        finished = true;
    } else if (h.slot < 0) {
        finished = true;                       // miss, or a traversal error
    } else {
        pt_ray r = path_ray(s);
        HitInfo hi; hi.t = h.t; hi.u = h.u; hi.v = h.v; hi.slot = h.slot;
        pt_flat_hit rec;
        finalize_hit(scene, r, hi, rec);
        if (p.debug == PT_DEBUG_NORMALS) { radiance = 0.5f * (mk(rec.normal) + mk(1, 1, 1)); finished = true; }
        else if (p.debug == PT_DEBUG_TRIANGLE) {
            radiance = rec.primitive_type == PT_TRIANGLE ? id_color(rec.primitive_id) : mk(0.3f, 0.3f, 0.3f);
            finished = true;
        } else if (p.debug == PT_DEBUG_MATERIAL) { radiance = id_color(rec.material_id); finished = true; }
        else {
            const pt_material mat = scene.materials[rec.material_id];
            f3 in_dir = mk(s.dx, s.dy, s.dz);
            f3 pos = mk(rec.p), normal = mk(rec.normal);
            if (mat.type == PT_LIGHT) {
                float weight = s.prev_pdf > 0 ? mis_weight(s.prev_pdf, hit_light_pdf(scene, mk(s.ox, s.oy, s.oz), rec)) : 1;
                radiance = radiance + weight * throughput * trace_texture(scene, mat.texture_id, rec.u, rec.v);
                finished = true;
            } else if (s.depth == p.max_depth) {
                finished = true;
            } else if (p.mis && mat.type == PT_DIFFUSE) {
                f3 attenuation = trace_texture(scene, mat.texture_id, rec.u, rec.v);
                if (scene.light_count) {
                    LightSample light = sample_light(scene, rng);
                    f3 delta = light.point - pos;
                    float distance = length(delta);
                    if (distance > 0.002f && finite(distance)) {
                        f3 direction = delta / distance;
                        float cosine = fmaxf(0, dot(normal, direction));
                        float pdf = light_direction_pdf(scene.light_area, pos, light.point, light.normal);
                        if (cosine > 0 && pdf > 0) {
                            const pt_material &emitter = scene.materials[light.material];
                            f3 emission = trace_texture(scene, emitter.texture_id, light.u, light.v);
                            float bsdf_pdf = cosine / float(M_PI);
                            f3 c = throughput * attenuation * emission * (bsdf_pdf * mis_weight(pdf, bsdf_pdf) / pdf);
                            sr.ox = pos.x; sr.oy = pos.y; sr.oz = pos.z; sr.tmax = distance - 0.001f;
                            sr.dx = direction.x; sr.dy = direction.y; sr.dz = direction.z; sr.time = s.time;
                            sr.cr = c.x; sr.cg = c.y; sr.cb = c.z; sr.pixel = slot;
                            shadow = true;
                        }
                    }
                }
                f3 direction = cosine_direction(normal, rng);
                s.prev_pdf = fmaxf(0, dot(normal, direction)) / float(M_PI);
                throughput = throughput * attenuation;
                s.ox = pos.x; s.oy = pos.y; s.oz = pos.z;
                s.dx = direction.x; s.dy = direction.y; s.dz = direction.z;
                s.depth++;
            } else {
                s.prev_pdf = 0;
                f3 attenuation, dir;
                if (!trace_scatter(scene, mat, in_dir, rec, rng, attenuation, dir)) finished = true;
                else {
                    throughput = throughput * attenuation;
                    s.ox = pos.x; s.oy = pos.y; s.oz = pos.z;
                    s.dx = dir.x; s.dy = dir.y; s.dz = dir.z;
                    s.depth++;
                }
            }
        }
    }
    if (finished) {
        // accumulated += trace_pixel_sample(...) (src/cuda/cuda_renderer.cu:81)
        sum[0] = sum[0] + radiance.x; sum[1] = sum[1] + radiance.y; sum[2] = sum[2] + radiance.z;
        s.samples_left--;
        if (s.samples_left > 0) {
            int left = s.samples_left;
            camera_path(*p.camera, p.width, p.height, pixel, rng, s);
            s.samples_left = left;
            return true;
        }
        return false;
    }
    s.tr = throughput.x; s.tg = throughput.y; s.tb = throughput.z;
    s.rr = radiance.x; s.rg = radiance.y; s.rb = radiance.z;
    return true;
}

} // namespace ptb
