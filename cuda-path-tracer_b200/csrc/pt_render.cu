// pt_render.cu — wavefront MIS path tracer (sm_100a, built with --fmad=false).
//
// Replaces class cuda_renderer and its render_pixels megakernel (src/cuda/cuda_renderer.cu:64-240).
// The reference runs trace_pixel_sample's whole bounce loop in one thread per pixel.  Here a
// path's bounce loop is cut into three kernels that run over queues of live paths:
//   extend : closest hit of every queued path's ray,
//   shade  : the rest of one trace_color iteration (emission with MIS weight, next-event
//            estimation that emits a shadow ray, cosine or material scatter), and, when a
//            sample ends, its radiance added to the pixel sum and the pixel's next camera ray,
//   shadow : any-hit of the shadow rays; an unoccluded one adds its precomputed contribution.
// Exactly one path per pixel is in flight, so every pixel's PCG stream is consumed in the
// reference's order and every float is summed in the reference's order: with the same
// arithmetic (--fmad=false, the same CUDA math functions) the sums, RNG states and ray count
// equal the reference renderer's.
#include <cfloat>
#include <algorithm>
#include <cstring>
#include <vector>
#include "pt_api_common.h"
#include "pt_device.h"
#include "pt_wavefront.h"

using namespace ptb;

namespace ptb {

struct RenderParams {
    pt_camera camera;
    int width, height, max_depth, debug, mis, brute, wide;
    int32_t leaves;
    const int32_t *brute_order;
};

struct RenderBuffers {
    PathState *paths;
    PathHit *hits;
    uint2 *stats;           // per-path box/primitive counts (bvh / intersections views)
    ShadowRay *shadows;
    int32_t *queue[2];
    int32_t *shadow_queue;
    int32_t *counters;      // [0],[1]: path queues; [2],[3]: shadow queues of even and odd iterations
    unsigned long long *fetch;   // [0]: extend's item counter, [1],[2]: the shadow kernels' item counters, [3]: finish_pair's
    unsigned long long *rays;
    int32_t *error;
    float *sums;
    Pcg *rng;
};

__device__ inline void camera_path(const RenderParams &p, int32_t pixel, Pcg &rng, PathState &s) {
    camera_path(p.camera, p.width, p.height, pixel, rng, s);
}

// initialize_pixels (src/cuda/cuda_renderer.cu:64-68)
__global__ void init_pixels(float *sums, Pcg *rng, int32_t count, uint64_t seed) {
    int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    sums[3 * i] = 0; sums[3 * i + 1] = 0; sums[3 * i + 2] = 0;
    Pcg r; r.seed(seed, uint64_t(i));
    rng[i] = r;
}

// First camera ray of every pixel; queue 0 = all pixels in order.
__global__ void start_samples(RenderParams p, RenderBuffers b, int32_t count, int samples) {
    int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        b.counters[0] = count; b.counters[1] = 0; b.counters[2] = 0; b.counters[3] = 0;
        b.fetch[0] = 0; b.fetch[1] = 0; b.fetch[2] = 0; b.fetch[3] = 0;
    }
    if (i >= count) return;
    Pcg rng = b.rng[i];
    PathState s;
    camera_path(p, i, rng, s);
    s.samples_left = samples;
    b.rng[i] = rng;
    b.paths[i] = s;
    b.queue[0][i] = i;
}

// extend: closest hit of each queued path (trace_color's trace_world, transport.h:177-178)
__global__ void __launch_bounds__(256, 4) extend_kernel(DeviceScene scene, RenderParams p, RenderBuffers b, int parity, int min_active) {
    const int32_t n = b.counters[parity];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(b.rays, (unsigned long long)n);
        b.counters[parity ^ 1] = 0;      // the next queue fills during shade
        // this iteration's shadow slot (the previous iteration's shadow kernel, which may still
        // be running on the other stream, uses the other slot)
        b.counters[2 + parity] = 0;
        b.fetch[1 + parity] = 0;
    }
    const int32_t *queue = b.queue[parity];
    if (!p.brute && p.debug != PT_DEBUG_BVH && p.debug != PT_DEBUG_INTERSECTIONS) {
        auto get = [&](size_t k, pt_ray &r, float &lo, float &hi) { r = path_ray(b.paths[queue[k]]); lo = 0.001f; hi = FLT_MAX; };
        auto done = [&](size_t k, const WalkResult &w) {
            if (w.error) *b.error = 1;
            PathHit out;
            out.t = w.t; out.u = w.u; out.v = w.v;
            out.slot = w.error ? -2 : w.slot;
            b.hits[queue[k]] = out;
        };
        if (p.wide == 2) persistent_walk4_spec<false>(scene, size_t(n), &b.fetch[0], min_active, kTieLastLeaf, get, done);
        else if (p.wide) persistent_walk4<false>(scene, size_t(n), &b.fetch[0], min_active, kTieLastLeaf, get, done);
        else persistent_walk<false>(scene, size_t(n), &b.fetch[0], min_active, kTieLastLeaf, get, done);
        return;
    }
    const bool reference_order = p.debug == PT_DEBUG_BVH || p.debug == PT_DEBUG_INTERSECTIONS;
    for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int32_t i = queue[k];
        PathState s = b.paths[i];
        pt_ray r = path_ray(s);
        HitInfo h;
        uint32_t boxes = 0, prims = 0;
        int error = 0;
        bool hit;
        if (p.brute) hit = traverse_brute<false>(scene, p.brute_order, p.leaves, r, 0.001f, FLT_MAX, kTieLastNode, h, prims);
        else hit = traverse_reference(scene, r, 0.001f, FLT_MAX, kTieLastLeaf, h, boxes, prims, error);
        if (error) *b.error = 1;
        PathHit out;
        out.t = h.t; out.u = h.u; out.v = h.v; out.slot = (hit && !error) ? h.slot : (error ? -2 : -1);
        b.hits[i] = out;
        if (reference_order) b.stats[i] = make_uint2(boxes, prims);
    }
}

__device__ inline ShadeCtx shade_ctx(const RenderParams &p) {
    ShadeCtx c;
    c.camera = &p.camera; c.width = p.width; c.height = p.height; c.max_depth = p.max_depth;
    c.debug = p.debug; c.mis = p.mis;
    return c;
}

// shade: shade_path over the queue; live paths and shadow rays are appended (warp-aggregated)
__global__ void __launch_bounds__(256, 4) shade_kernel(DeviceScene scene, RenderParams p, RenderBuffers b, int parity) {
    const int32_t n = b.counters[parity];
    const int32_t *in = b.queue[parity];
    int32_t *out = b.queue[parity ^ 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) b.fetch[0] = 0;   // extend's item counter, for the next iteration
    for (int32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        int32_t k = base + threadIdx.x;
        bool valid = k < n;
        bool live = false, shadow = false;
        int32_t i = valid ? in[k] : 0;
        if (valid) {
            PathState s = b.paths[i];
            PathHit h = b.hits[i];
            uint2 st = (p.debug == PT_DEBUG_BVH || p.debug == PT_DEBUG_INTERSECTIONS) ? b.stats[i] : make_uint2(0, 0);
            Pcg rng = b.rng[i];
            ShadowRay sr;
            live = shade_path(scene, shade_ctx(p), b.sums + 3 * size_t(i), i, i, s, h, st, rng, sr, shadow);
            b.paths[i] = s;
            b.rng[i] = rng;
            if (shadow) b.shadows[i] = sr;
        }
        push(live, i, out, &b.counters[parity ^ 1]);
        push(shadow, i, b.shadow_queue, &b.counters[2 + parity]);
    }
}

// finish: the queue's remaining paths run to the end of their pixel's samples, one thread per
// path (the reference's megakernel form).  Used once the queue is short, where a wavefront
// iteration would cost the latency of its slowest ray for a handful of rays, on two-wide trees,
// with the brute-force walk, for the bvh / intersections views and on trees of at most 32
// four-wide nodes, which the renderer walks in the two-wide layout (otherwise finish_pair_kernel).
// walk forms the one-lane finish kernel rarely runs (brute force, the debug views' reference-order
// walk, four-wide trees outside the pair tail), called out of line so that the bounce loop's hot
// path stays compact in the instruction cache
template <bool kAny>
__device__ __noinline__ bool cold_brute(const DeviceScene &scene, const int32_t *order, int32_t leaves, const pt_ray &r, float tmax,
                                        HitInfo &h, uint32_t &prims) {
    return traverse_brute<kAny>(scene, order, leaves, r, 0.001f, tmax, kTieLastNode, h, prims);
}
__device__ __noinline__ bool cold_reference(const DeviceScene &scene, const pt_ray &r, HitInfo &h, uint32_t &boxes, uint32_t &prims,
                                            int &error) {
    return traverse_reference(scene, r, 0.001f, FLT_MAX, kTieLastLeaf, h, boxes, prims, error);
}
template <bool kAny>
__device__ __noinline__ bool cold_walk4(const DeviceScene &scene, const pt_ray &r, float tmax, HitInfo &h, uint32_t &boxes,
                                        uint32_t &prims, int &error) {
    return traverse4<kAny>(scene, r, 0.001f, tmax, kTieLastLeaf, h, boxes, prims, error);
}

__global__ void finish_kernel(DeviceScene scene, RenderParams p, RenderBuffers b, int parity) {
    const int32_t n = b.counters[parity];
    const bool reference_order = p.debug == PT_DEBUG_BVH || p.debug == PT_DEBUG_INTERSECTIONS;
    unsigned long long rays = 0;
    for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int32_t i = b.queue[parity][k];
        PathState s = b.paths[i];
        Pcg rng = b.rng[i];
        for (;;) {
            rays++;   // each closest-hit query counts once, as trace_color counts it (transport.h:177)
            pt_ray r = path_ray(s);
            HitInfo hi;
            uint32_t boxes = 0, prims = 0;
            int error = 0;
            bool hit;
            if (p.brute) hit = cold_brute<false>(scene, p.brute_order, p.leaves, r, FLT_MAX, hi, prims);
            else if (reference_order) hit = cold_reference(scene, r, hi, boxes, prims, error);
            else if (p.wide) hit = cold_walk4<false>(scene, r, FLT_MAX, hi, boxes, prims, error);
            else hit = traverse<false>(scene, r, 0.001f, FLT_MAX, kTieLastLeaf, hi, boxes, prims, error);
            if (error) *b.error = 1;
            PathHit h;
            h.t = hi.t; h.u = hi.u; h.v = hi.v; h.slot = (hit && !error) ? hi.slot : (error ? -2 : -1);
            ShadowRay sr;
            bool shadow = false;
            bool live = shade_path(scene, shade_ctx(p), b.sums + 3 * size_t(i), i, i, s, h, make_uint2(boxes, prims), rng, sr, shadow);
            if (shadow) {
                rays++;
                pt_ray q;
                q.origin = pt_vec3{sr.ox, sr.oy, sr.oz};
                q.direction = pt_vec3{sr.dx, sr.dy, sr.dz};
                q.time = sr.time;
                HitInfo sh;
                uint32_t sb = 0, spr = 0;
                int serr = 0;
                bool blocked = p.brute ? cold_brute<true>(scene, p.brute_order, p.leaves, q, sr.tmax, sh, spr)
                             : p.wide ? cold_walk4<true>(scene, q, sr.tmax, sh, sb, spr, serr)
                                      : traverse<true>(scene, q, 0.001f, sr.tmax, kTieLastLeaf, sh, sb, spr, serr);
                if (serr) *b.error = 1;
                else if (!blocked) { s.rr = s.rr + sr.cr; s.rg = s.rg + sr.cg; s.rb = s.rb + sr.cb; }
            }
            if (!live) break;
        }
        b.paths[i] = s;
        b.rng[i] = rng;
    }
    // one add per warp
    for (int o = 16; o; o >>= 1) rays += __shfl_down_sync(0xffffffffu, rays, o);
    if ((threadIdx.x & 31) == 0 && rays) atomicAdd(b.rays, rays);
}

// finish, two lanes per path (four-wide tree, shading views): in each round the even lane of a
// pair walks the path's next extension ray while the odd lane walks the shadow ray of the path's
// previous bounce.  A shadow ray only adds to the radiance and the extension ray depends on
// neither, so a bounce costs one walk's latency instead of two, and both walks run the same
// instructions (traverse4_rt).  The shadow contribution of bounce k is added before bounce k+1
// is shaded, as in the one-lane form, so sums, ray counts and streams are bit-identical.  A pair
// whose path has ended takes the next queue entry from fetch[3] (zeroed before the launch).
__global__ void __launch_bounds__(256, 2) finish_pair_kernel(DeviceScene scene, RenderParams p, RenderBuffers b, int parity) {
    const int32_t n = b.counters[parity];
    const unsigned full = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31;
    const bool odd = lane & 1;
    const unsigned even_lane = lane & ~1u, odd_lane = lane | 1u;
    unsigned long long rays = 0;
    int32_t i = -1;                // even lane: the path (slot) in hand, -1 when none
    PathState s{};
    Pcg rng{};
    bool live = false;             // even lane: the path has an extension ray to walk
    bool pending = false;          // even lane: a shadow ray from the last shading waits
    bool drained = false;          // even lane: the queue had no entry left for this pair
    ShadowRay sr{};
    bool walk_shadow = false;      // odd lane: walks the pair's pending shadow ray this round
    pt_ray q{};
    float qmax = 0;
    for (;;) {
        if (!odd && !live && !pending && !drained) {
            if (i >= 0) { b.paths[i] = s; b.rng[i] = rng; i = -1; }
            unsigned long long k = atomicAdd(&b.fetch[3], 1ull);
            if (k < (unsigned long long)n) {
                i = b.queue[parity][k];
                s = b.paths[i];
                rng = b.rng[i];
                live = true;
            } else {
                drained = true;
            }
        }
        const bool work = odd ? walk_shadow : live;   // both lanes' rounds stay in step (warp-uniform loop)
        if (!__any_sync(full, work)) break;
        HitInfo hi;
        uint32_t boxes = 0, prims = 0;
        int error = 0;
        bool hit = false;
        if (work) {
            rays++;   // each query counts once, as trace_color counts it (transport.h:177)
            hit = traverse4_rt(scene, odd ? q : path_ray(s), 0.001f, odd ? qmax : FLT_MAX, kTieLastLeaf, odd, hi, boxes,
                               prims, error);
        }
        const bool blocked = __shfl_sync(full, hit, odd_lane);
        const int shadow_error = __shfl_sync(full, error, odd_lane);
        if (!odd) {
            if (pending) {
                if (shadow_error) *b.error = 1;
                else if (!blocked) { s.rr = s.rr + sr.cr; s.rg = s.rg + sr.cg; s.rb = s.rb + sr.cb; }
                pending = false;
            }
            if (live) {
                if (error) *b.error = 1;
                PathHit h;
                h.t = hi.t; h.u = hi.u; h.v = hi.v; h.slot = (hit && !error) ? hi.slot : (error ? -2 : -1);
                bool shadow = false;
                live = shade_path(scene, shade_ctx(p), b.sums + 3 * size_t(i), i, i, s, h, make_uint2(boxes, prims), rng, sr, shadow);
                pending = shadow;
            }
        }
        // the even lane hands its new shadow ray to the odd lane
        walk_shadow = __shfl_sync(full, pending, even_lane);
        q.origin.x = __shfl_sync(full, sr.ox, even_lane);
        q.origin.y = __shfl_sync(full, sr.oy, even_lane);
        q.origin.z = __shfl_sync(full, sr.oz, even_lane);
        q.direction.x = __shfl_sync(full, sr.dx, even_lane);
        q.direction.y = __shfl_sync(full, sr.dy, even_lane);
        q.direction.z = __shfl_sync(full, sr.dz, even_lane);
        q.time = __shfl_sync(full, sr.time, even_lane);
        qmax = __shfl_sync(full, sr.tmax, even_lane);
    }
    if (!odd && i >= 0) { b.paths[i] = s; b.rng[i] = rng; }
    for (int o = 16; o; o >>= 1) rays += __shfl_down_sync(full, rays, o);
    if (lane == 0 && rays) atomicAdd(b.rays, rays);
}

// shadow: any-hit of the NEE rays (transport.h:206-214); unoccluded ones add their contribution
__global__ void __launch_bounds__(256, 4) shadow_kernel(DeviceScene scene, RenderParams p, RenderBuffers b, int parity, int min_active) {
    const int32_t n = b.counters[2 + parity];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(b.rays, (unsigned long long)n);
    auto add = [&](int32_t i, const ShadowRay &sr) {
        PathState &s = b.paths[i];
        s.rr = s.rr + sr.cr; s.rg = s.rg + sr.cg; s.rb = s.rb + sr.cb;
    };
    if (!p.brute) {
        auto get = [&](size_t k, pt_ray &r, float &lo, float &hi) {
            const ShadowRay &sr = b.shadows[b.shadow_queue[k]];
            r.origin = pt_vec3{sr.ox, sr.oy, sr.oz};
            r.direction = pt_vec3{sr.dx, sr.dy, sr.dz};
            r.time = sr.time;
            lo = 0.001f; hi = sr.tmax;
        };
        auto done = [&](size_t k, const WalkResult &w) {
            if (w.error) { *b.error = 1; return; }
            if (w.slot < 0) { int32_t i = b.shadow_queue[k]; add(i, b.shadows[i]); }
        };
        if (p.wide == 2) persistent_walk4_spec<true>(scene, size_t(n), &b.fetch[1 + parity], min_active, kTieLastLeaf, get, done);
        else if (p.wide) persistent_walk4<true>(scene, size_t(n), &b.fetch[1 + parity], min_active, kTieLastLeaf, get, done);
        else persistent_walk<true>(scene, size_t(n), &b.fetch[1 + parity], min_active, kTieLastLeaf, get, done);
        return;
    }
    for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int32_t i = b.shadow_queue[k];
        ShadowRay sr = b.shadows[i];
        pt_ray r;
        r.origin = pt_vec3{sr.ox, sr.oy, sr.oz};
        r.direction = pt_vec3{sr.dx, sr.dy, sr.dz};
        r.time = sr.time;
        HitInfo h;
        uint32_t prims = 0;
        bool blocked = traverse_brute<true>(scene, p.brute_order, p.leaves, r, 0.001f, sr.tmax, kTieLastNode, h, prims);
        if (!blocked) add(i, sr);
    }
}

// pack_pixels (src/cuda/cuda_renderer.cu:99-109)
__global__ void pack_pixels(const float *sum, unsigned char *rgba, size_t count, int samples) {
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    f3 color = samples ? mk(sum[3 * i], sum[3 * i + 1], sum[3 * i + 2]) / float(samples) : mk(0, 0, 0);
    for (int channel = 0; channel < 3; channel++) {
        float value = comp(color, channel);
        float gamma = value > 0 && value < 1 ? sqrtf(value) : 0;
        rgba[4 * i + channel] = !(value > 0) ? 0 : value >= 1 ? 255 : int(255.99 * gamma);
    }
    rgba[4 * i + 3] = 255;
}

// shared-memory stack of the persistent walks (the larger of the two layouts' needs)
size_t stack_bytes(int block) {
    return std::max(size_t(kSharedStack) * sizeof(int32_t), size_t(kSharedStack4) * sizeof(int2)) * size_t(block);
}

// The one-lane finish kernel runs in blocks of 128: its paths then spread evenly over the SMs
// (config 1, all 64,000 paths in the tail: 7.2 -> 6.8 ms against blocks of 256, two per SM on
// 102 SMs and one on the rest).
constexpr int kFinishBlock = 128;

int occupancy_grid(const void *kernel, int block, size_t smem = 0) {
    int per_sm = 0;
    PT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem));
    return device_sm_count() * (per_sm > 0 ? per_sm : 1);
}

} // namespace ptb

struct pt_renderer {
    const pt_scene *scene = nullptr;
    RenderParams params{};
    uint64_t seed = 0;
    int32_t pixels = 0;
    int samples = 0;
    float milliseconds = 0;
    uint64_t rays = 0;
    // threads per block of the wavefront kernels (pt_set_block_shape): 16x8 by default (config 2:
    // 64.3 ms per render against 65.1 with the reference's 16x16; config 1 unchanged)
    int block = 128;
    int grid_extend = 0, grid_shade = 0, grid_shadow = 0, grid_finish = 0, grid_finish_pair = 0;
    int32_t tail_paths = 0;             // live-path count below which the fused finish kernel takes over
    bool pair_tail = false;             // the tail runs two lanes per path (finish_pair_kernel)
    DeviceBuffer paths, hits, stats, shadows, queue0, queue1, shadow_queue, counters, fetch, ray_total, error, sums, rng, rgba;
    RenderBuffers buf{};
    cudaStream_t stream = nullptr;
    cudaStream_t shadow_stream = nullptr;   // shadow kernel k runs beside extend k+1
    Event start, stop;
    Event shaded[2], shadowed[2];           // by iteration parity
    int32_t *host_counters = nullptr;   // pinned, one slot per in-flight iteration
    Event iteration_events[8];
    ~pt_renderer() {
        if (host_counters) cudaFreeHost(host_counters);
        if (shadow_stream) cudaStreamDestroy(shadow_stream);
        if (stream) cudaStreamDestroy(stream);
    }
    void grids() {
        grid_extend = occupancy_grid((const void *)extend_kernel, block, stack_bytes(block));
        grid_shade = occupancy_grid((const void *)shade_kernel, block);
        grid_shadow = occupancy_grid((const void *)shadow_kernel, block, stack_bytes(block));
        grid_finish = occupancy_grid((const void *)finish_kernel, kFinishBlock);
        grid_finish_pair = occupancy_grid((const void *)finish_pair_kernel, block);
    }
};

namespace {
void validate_camera(const pt_camera &c) {
    // validate_render_camera, src/renderer/render_validation.h:16-22
    for (const pt_vec3 &v : {c.origin, c.lower_left_corner, c.horizontal, c.vertical, c.u, c.v})
        if (!std::isfinite(v.x) || !std::isfinite(v.y) || !std::isfinite(v.z))
            throw Error(PT_INVALID_ARGUMENT, "camera contains nonfinite values");
    if (!std::isfinite(c.lens_radius) || c.lens_radius < 0 || !std::isfinite(c.time0) || !std::isfinite(c.time1) || c.time1 < c.time0)
        throw Error(PT_INVALID_ARGUMENT, "invalid camera lens/shutter");
}
constexpr int kIterationRing = 8;   // == size of pt_renderer::iteration_events
} // namespace

extern "C" {

pt_status pt_renderer_create(const pt_scene *scene, const pt_camera *camera, int width, int height, uint64_t seed,
                             uint32_t flags, int debug_mode, int max_depth, pt_renderer **out) {
    return guard([&]() {
        if (!scene || !camera || !out) throw Error(PT_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        // checked_pixel_count and validate_render_mode (src/renderer/render_validation.h:7-15)
        if (width <= 0 || height <= 0 || uint64_t(width) * uint64_t(height) > uint64_t(INT32_MAX))
            throw Error(PT_INVALID_ARGUMENT, "image dimensions exceed supported pixel count");
        if (debug_mode < PT_DEBUG_SHADED || debug_mode > PT_DEBUG_INTERSECTIONS) throw Error(PT_INVALID_ARGUMENT, "invalid render debug mode");
        if (max_depth < 0 || max_depth > 100000) throw Error(PT_INVALID_ARGUMENT, "invalid bounce limit");
        validate_camera(*camera);
        require_device();
        auto r = new pt_renderer;
        try {
            size_t n = size_t(width) * size_t(height);
            r->scene = scene;
            r->seed = seed;
            r->pixels = int32_t(n);
            RenderParams &p = r->params;
            p.camera = *camera; p.width = width; p.height = height; p.max_depth = max_depth;
            p.debug = debug_mode; p.mis = (flags & PT_RENDER_MIS) ? 1 : 0; p.brute = (flags & PT_RENDER_BRUTE) ? 1 : 0;
            p.leaves = scene->leaf_count; p.brute_order = scene->brute_order.get<int32_t>();
            p.wide = (g_query_config.wide && scene->view.nodes4) ? (g_query_config.speculative ? 2 : 1) : 0;
            r->paths.resize(n * sizeof(PathState));
            r->hits.resize(n * sizeof(PathHit));
            if (debug_mode == PT_DEBUG_BVH || debug_mode == PT_DEBUG_INTERSECTIONS) r->stats.resize(n * sizeof(uint2));
            r->shadows.resize(n * sizeof(ShadowRay));
            r->queue0.resize(n * sizeof(int32_t));
            r->queue1.resize(n * sizeof(int32_t));
            r->shadow_queue.resize(n * sizeof(int32_t));
            r->counters.resize(4 * sizeof(int32_t));
            r->fetch.resize(4 * sizeof(unsigned long long));
            r->ray_total.resize(sizeof(unsigned long long));
            r->error.resize(sizeof(int32_t));
            r->sums.resize(n * 3 * sizeof(float));
            r->rng.resize(n * sizeof(Pcg));
            RenderBuffers &b = r->buf;
            b.paths = r->paths.get<PathState>(); b.hits = r->hits.get<PathHit>(); b.stats = r->stats.get<uint2>();
            b.shadows = r->shadows.get<ShadowRay>();
            b.queue[0] = r->queue0.get<int32_t>(); b.queue[1] = r->queue1.get<int32_t>();
            b.shadow_queue = r->shadow_queue.get<int32_t>(); b.counters = r->counters.get<int32_t>();
            b.fetch = r->fetch.get<unsigned long long>();
            b.rays = r->ray_total.get<unsigned long long>(); b.error = r->error.get<int32_t>();
            b.sums = r->sums.get<float>(); b.rng = r->rng.get<Pcg>();
            PT_CUDA(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
            PT_CUDA(cudaStreamCreateWithFlags(&r->shadow_stream, cudaStreamNonBlocking));
            PT_CUDA(cudaMallocHost(&r->host_counters, kIterationRing * sizeof(int32_t)));
            r->grids();
            // below 65,536 live paths the fused kernel holds them all at once (measured: config 1 is 3.6 %
            // faster than with a floor of 16,384; larger images are unchanged)
            r->tail_paths = std::max<int32_t>(65536, r->pixels / 4);
            // On a tree of a few nodes (tens of primitives) a bounce is mostly shading: the two-wide walk
            // (fewer instructions per visit) and one lane per path in the tail are faster there
            // (config 1, 23 primitives: 8.4 ms per render with the four-wide walk and two lanes per
            // path, 6.8 with one lane, 6.5 with the two-wide walk too); from a few hundred triangles on,
            // two lanes per path win (772 triangles: 3.4 vs 4.1 ms).
            constexpr size_t kSmallTreeNodes = 32;
            if (p.wide && scene->nodes4.bytes() / sizeof(Bvh4QNode) <= kSmallTreeNodes) p.wide = 0;
            r->pair_tail = p.wide != 0;
        } catch (...) { delete r; throw; }
        *out = r;
        pt_status st = pt_reset(r, camera);
        if (st != PT_OK) { delete r; *out = nullptr; throw Error(st, pt_last_error()); }
    });
}

pt_status pt_renderer_destroy(pt_renderer *r) { delete r; return PT_OK; }

// reset(camera) (src/cuda/cuda_renderer.cu:186-194)
pt_status pt_reset(pt_renderer *r, const pt_camera *camera) {
    return guard([&]() {
        if (!r || !camera) throw Error(PT_INVALID_ARGUMENT, "null argument");
        validate_camera(*camera);
        PT_CUDA(cudaMemsetAsync(r->buf.error, 0, sizeof(int32_t), r->stream));
        init_pixels<<<(r->pixels + 255) / 256, 256, 0, r->stream>>>(r->buf.sums, r->buf.rng, r->pixels, r->seed);
        PT_CUDA(cudaGetLastError());
        PT_CUDA(cudaStreamSynchronize(r->stream));
        r->params.camera = *camera;
        r->samples = 0; r->milliseconds = 0; r->rays = 0;
    });
}

// add_samples(count) (src/cuda/cuda_renderer.cu:196-213)
pt_status pt_add_samples(pt_renderer *r, int count) {
    return guard([&]() {
        if (!r) throw Error(PT_INVALID_ARGUMENT, "null renderer");
        if (count <= 0 || count > INT32_MAX - r->samples) throw Error(PT_INVALID_ARGUMENT, "invalid accumulated sample count");
        const DeviceScene &scene = r->scene->view;
        cudaStream_t st = r->stream;
        PT_CUDA(cudaMemsetAsync(r->buf.rays, 0, sizeof(unsigned long long), st));
        PT_CUDA(cudaEventRecord(r->start.get(), st));
        start_samples<<<(r->pixels + 255) / 256, 256, 0, st>>>(r->params, r->buf, r->pixels, count);
        PT_CUDA(cudaGetLastError());
        // Every pixel needs at most count * (max_depth + 1) extends; the loop ends earlier when
        // the queue is empty.  The queue length is read back with a lag of a few iterations.
        // Iteration k: extend k and shade k on the main stream, shadow k on the shadow stream
        // after shade k; shade k+1 waits for shadow k (it rewrites the shadow records and reads
        // the radiance shadow k adds), so shadow k overlaps extend k+1 only.
        const int64_t max_iterations = int64_t(count) * (int64_t(r->params.max_depth) + 1) + 1;
        int parity = 0;
        int64_t issued = 0, checked = 0;
        bool done = false, tail = false;
        while (!done && !tail && issued < max_iterations) {
            extend_kernel<<<r->grid_extend, r->block, stack_bytes(r->block), st>>>(scene, r->params, r->buf, parity, g_query_config.min_active);
            if (issued > 0) PT_CUDA(cudaStreamWaitEvent(st, r->shadowed[parity ^ 1].get(), 0));
            shade_kernel<<<r->grid_shade, r->block, 0, st>>>(scene, r->params, r->buf, parity);
            PT_CUDA(cudaEventRecord(r->shaded[parity].get(), st));
            PT_CUDA(cudaStreamWaitEvent(r->shadow_stream, r->shaded[parity].get(), 0));
            shadow_kernel<<<r->grid_shadow, r->block, stack_bytes(r->block), r->shadow_stream>>>(scene, r->params, r->buf, parity,
                                                                                                  g_query_config.min_active);
            PT_CUDA(cudaEventRecord(r->shadowed[parity].get(), r->shadow_stream));
            PT_CUDA(cudaGetLastError());
            parity ^= 1;
            int slot = int(issued % kIterationRing);
            PT_CUDA(cudaMemcpyAsync(&r->host_counters[slot], &r->buf.counters[parity], sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            PT_CUDA(cudaEventRecord(r->iteration_events[slot].get(), st));
            issued++;
            // keep at most kIterationRing/2 iterations ahead of the last one inspected
            while (checked < issued && (issued - checked >= kIterationRing / 2 ||
                                        cudaEventQuery(r->iteration_events[int(checked % kIterationRing)].get()) == cudaSuccess)) {
                PT_CUDA(cudaEventSynchronize(r->iteration_events[int(checked % kIterationRing)].get()));
                int32_t live = r->host_counters[int(checked % kIterationRing)];
                if (live == 0) { done = true; break; }
                if (live < r->tail_paths) { tail = true; break; }
                checked++;
            }
        }
        // the last shadow kernel joins the main stream
        if (issued > 0) PT_CUDA(cudaStreamWaitEvent(st, r->shadowed[parity ^ 1].get(), 0));
        if (tail && !done) {
            // the few remaining paths (of the last issued iteration's queue) run to completion
            const RenderParams &q = r->params;
            if (r->pair_tail && !q.brute && q.debug != PT_DEBUG_BVH && q.debug != PT_DEBUG_INTERSECTIONS) {
                PT_CUDA(cudaMemsetAsync(&r->buf.fetch[3], 0, sizeof(unsigned long long), st));
                finish_pair_kernel<<<r->grid_finish_pair, r->block, 0, st>>>(scene, q, r->buf, parity);
            } else
                finish_kernel<<<r->grid_finish, kFinishBlock, 0, st>>>(scene, q, r->buf, parity);
            PT_CUDA(cudaGetLastError());
            done = true;
        }
        while (!done && checked < issued) {   // iterations issued but not yet inspected
            PT_CUDA(cudaEventSynchronize(r->iteration_events[int(checked % kIterationRing)].get()));
            if (r->host_counters[int(checked % kIterationRing)] == 0) done = true;
            checked++;
        }
        PT_CUDA(cudaEventRecord(r->stop.get(), st));
        PT_CUDA(cudaEventSynchronize(r->stop.get()));
        int32_t error = 0;
        unsigned long long total = 0;
        PT_CUDA(cudaMemcpy(&error, r->buf.error, sizeof error, cudaMemcpyDeviceToHost));
        if (error) throw Error(PT_STACK_OVERFLOW, "CUDA traversal stack overflow");
        if (!done) throw Error(PT_TIMEOUT, "wavefront did not drain within its iteration bound");
        float ms = 0;
        PT_CUDA(cudaEventElapsedTime(&ms, r->start.get(), r->stop.get()));
        PT_CUDA(cudaMemcpy(&total, r->buf.rays, sizeof total, cudaMemcpyDeviceToHost));
        r->milliseconds += ms;
        r->samples += count;
        r->rays += total;
    });
}

// Live-path count below which add_samples hands the remaining paths to the fused finish kernel
// (0: wavefront to the end; INT32_MAX: fused kernel from the first iteration).
pt_status pt_renderer_tuning(pt_renderer *r, int32_t tail_paths) {
    return guard([&]() {
        if (!r || tail_paths < 0) throw Error(PT_INVALID_ARGUMENT, "invalid renderer tuning");
        r->tail_paths = tail_paths;
    });
}

// set_block_shape (src/cuda/cuda_renderer.cu:215-228): the accepted shapes, as block sizes.
pt_status pt_set_block_shape(pt_renderer *r, int width, int height) {
    return guard([&]() {
        if (!r) throw Error(PT_INVALID_ARGUMENT, "null renderer");
        if (!((width == 8 && height == 8) || (width == 16 && height == 8) || (width == 16 && height == 16) || (width == 32 && height == 8)))
            throw Error(PT_INVALID_ARGUMENT, "CUDA block must be 8x8, 16x8, 16x16 or 32x8");
        r->block = width * height;
        r->grids();
    });
}

pt_status pt_get_sums(const pt_renderer *r, float *rgb, size_t floats) {
    return guard([&]() {
        if (!r || !rgb || floats < size_t(r->pixels) * 3) throw Error(PT_INVALID_ARGUMENT, "sum buffer too small");
        PT_CUDA(cudaMemcpy(rgb, r->buf.sums, size_t(r->pixels) * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

// image(): sums scaled by vec3::operator/= (reciprocal taken in double), on the host like the reference
pt_status pt_get_image(const pt_renderer *r, float *rgb, size_t floats) {
    return guard([&]() {
        pt_status st = pt_get_sums(r, rgb, floats);
        if (st != PT_OK) throw Error(st, pt_last_error());
        if (!r->samples) return;
        float k = (float)(1.0 / (double)float(r->samples));
        for (size_t i = 0; i < size_t(r->pixels) * 3; i++) rgb[i] *= k;
    });
}

pt_status pt_get_rng(const pt_renderer *r, uint64_t *words, size_t count) {
    return guard([&]() {
        if (!r || !words || count < size_t(r->pixels) * 2) throw Error(PT_INVALID_ARGUMENT, "rng buffer too small");
        PT_CUDA(cudaMemcpy(words, r->buf.rng, size_t(r->pixels) * sizeof(Pcg), cudaMemcpyDeviceToHost));
    });
}

pt_status pt_write_rgba(const pt_renderer *r, unsigned char *device_pixels, size_t bytes) {
    return guard([&]() {
        if (!r) throw Error(PT_INVALID_ARGUMENT, "null renderer");
        size_t count = size_t(r->pixels);
        if (!device_pixels || bytes < 4 * count) throw Error(PT_INVALID_ARGUMENT, "CUDA RGBA destination is too small");
        pack_pixels<<<unsigned((count + 255) / 256), 256, 0, r->stream>>>(r->buf.sums, device_pixels, count, r->samples);
        PT_CUDA(cudaGetLastError());
        PT_CUDA(cudaStreamSynchronize(r->stream));
    });
}

pt_status pt_rgba_image(const pt_renderer *cr, unsigned char *host_pixels, size_t bytes) {
    return guard([&]() {
        pt_renderer *r = const_cast<pt_renderer *>(cr);
        if (!r) throw Error(PT_INVALID_ARGUMENT, "null renderer");
        size_t count = size_t(r->pixels);
        if (!host_pixels || bytes < 4 * count) throw Error(PT_INVALID_ARGUMENT, "RGBA destination is too small");
        r->rgba.reserve(4 * count);
        pt_status st = pt_write_rgba(r, r->rgba.get<unsigned char>(), 4 * count);
        if (st != PT_OK) throw Error(st, pt_last_error());
        PT_CUDA(cudaMemcpy(host_pixels, r->rgba.get(), 4 * count, cudaMemcpyDeviceToHost));
    });
}

pt_status pt_stats(const pt_renderer *r, int *samples, float *kernel_ms, uint64_t *rays) {
    return guard([&]() {
        if (!r) throw Error(PT_INVALID_ARGUMENT, "null renderer");
        if (samples) *samples = r->samples;
        if (kernel_ms) *kernel_ms = r->milliseconds;
        if (rays) *rays = r->rays;
    });
}

} // extern "C"
