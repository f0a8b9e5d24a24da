// pt_cache_render.cu — path tracing with the learned radiance cache (sm_100a).
//
// No counterpart in the reference (its renderer has no learned component); the shading is the
// reference's MIS bounce loop (src/renderer/transport.h:169-230) as pt_wavefront.h has it.
//
// One frame = `samples_per_frame` samples per pixel, one path per pixel at a time (a pixel's
// next sample starts when its path ends), run as a wavefront:
//   start   : camera ray of every pixel (training-only frames: of the training pixels only);
//             about `training_paths` pixels, picked by a hash of (seed, frame, pixel), also
//             get a training slot for their first sample;
//   extend / shade / shadow, in pairs, while at least `tail_paths` paths are live (a device-
//             side WHILE loop in the frame's graph), then one fused kernel (a thread per path)
//             runs the short tail to its end:
//             shade does the MIS step, tracks the path's area spread
//               a0 = |x0 - x1|^2 / (4 pi cos1),  sqrt(a) += sqrt(|x_{i-1} - x_i|^2 / (pdf_{i-1} cos_i)),
//             and at the first diffuse vertex (past the primary hit) where a > c * a0 it ends the
//             path with a cache query (pixel gets radiance + throughput * albedo * prediction).
//             A training path instead records that vertex and the diffuse vertices of the next
//             `suffix_bounces` bounces (features, suffix radiance S and suffix throughput U as
//             seen there), and ends with a cache query at the vertex after them (self-training);
//   forward : the network on every query of the frame (tcgen05, pt_mlp.cu);
//   resolve : pixel sums += weight * prediction of each of the pixel's queries (in sample order;
//             the radiance before the query was added when the sample ended);
//   targets : for each recorded vertex, L = (S_end + U_end * albedo_tail * prediction - S_v) / U_v
//             is the outgoing radiance there; the sample (features, L / albedo) goes to one of
//             `train_steps` batches;
//   train   : one Adam step per batch.
// The launch sequence of a frame is fixed (queue lengths stay on the device), so a frame is
// captured once as a CUDA graph and replayed.
#include <cfloat>
#include <algorithm>
#include <cmath>
#include <vector>
#include "pt_api_common.h"
#include "pt_cache_internal.h"
#include "pt_device.h"
#include "pt_wavefront.h"

using namespace ptb;

namespace ptb {
size_t stack_bytes(int block);                                  // pt_render.cu
int occupancy_grid(const void *kernel, int block, size_t smem);  // pt_render.cu

namespace nrc {

constexpr int kMaxSuffix = 8;
constexpr int kMaxSteps = 8;
constexpr int kShadowSlot = 5 + kMaxSteps;   // counters[kShadowSlot + parity]: shadow queue of even / odd iterations
constexpr int kCounters = kShadowSlot + 2;

struct alignas(16) CachePath {
    float ox, oy, oz, time;
    float dx, dy, dz, bounce_pdf;       // bounce_pdf: density of this direction at the ray's origin (0: camera or specular)
    float tr, tg, tb, prev_pdf;         // throughput from the camera; MIS pdf of the last diffuse bounce
    float rr, rg, rb, spread;           // radiance so far; running sum of sqrt(footprint) terms
    float ur, ug, ub, a0;               // suffix throughput (training paths); primary footprint
    float sr, sg, sb; int32_t depth;    // suffix radiance (training paths)
    int32_t train;                      // training slot, -1: none
    int32_t vertices;                   // training vertices recorded, -1: the query vertex not reached yet
    int32_t qdepth;                     // depth of the query vertex
    int32_t samples_left;               // this one included
};
static_assert(sizeof(CachePath) == 112, "path record");

struct alignas(16) CacheShadow {
    float ox, oy, oz, tmax;
    float dx, dy, dz, time;
    float cr, cg, cb; int32_t path;     // contribution to the pixel
    float sr, sg, sb; int32_t suffix;   // contribution to the suffix radiance (suffix != 0)
};
static_assert(sizeof(CacheShadow) == 64, "shadow record");

struct alignas(16) QueryAux { float wr, wg, wb; int32_t path; };   // pixel weight of the prediction

struct alignas(16) TrainVertex {
    pt_cache_query q;
    float sr, sg, sb;                   // suffix radiance before the vertex's own estimate
    float ur, ug, ub;                   // suffix throughput at the vertex
    float pad;
};
static_assert(sizeof(TrainVertex) == 80, "training vertex record");

struct alignas(16) TrainEnd {
    float sr, sg, sb; int32_t query;    // suffix radiance at the end; tail query (-1: none)
    float wr, wg, wb; int32_t vertices; // suffix throughput x tail albedo
};

struct Params {
    pt_camera camera;
    int width, height, max_depth, wide;
    int use_cache, suffix_bounces, steps, accumulate, query_specular;
    int spf;                            // samples per pixel in this frame
    float spread_c;
    uint32_t train_threshold;           // a pixel trains when its hash is below this
    int32_t train_capacity;             // training slots
    int32_t bucket_capacity;            // samples per Adam step
    uint64_t seed;
    float radiance_max[3];              // brightest emitted radiance per channel: bounds every L / albedo
};

struct Buffers {
    CachePath *paths;
    PathHit *hits;
    CacheShadow *shadows;
    int32_t *queue[2];
    int32_t *shadow_queue;
    int32_t *counters;                  // [0],[1] path queues, [2] shadow queue, [3] queries, [4] training slots, [5..) batch sizes
    unsigned long long *fetch;          // item counters: [0] extend, [1],[2] shadow, [3] finish_pair
    unsigned long long *totals;         // [0] rays, [1] queries, [2] training samples
    int32_t *error;
    float *sums;
    Pcg *rng;
    uint32_t *frame;
    unsigned long long *pairs;          // wavefront iteration pairs run in this frame
    pt_cache_query *queries;
    QueryAux *aux;
    float *pred;
    int32_t *pixel_queries;             // pixel i's queries of the frame, in sample order: [i * spf + j]
    int32_t *pixel_query_count;
    TrainVertex *vertices;
    TrainEnd *ends;
    pt_cache_query *samples;            // steps x bucket_capacity
    float *targets;                     // steps x bucket_capacity x 3
};

__device__ inline uint32_t pixel_hash(uint64_t seed, uint32_t frame, int32_t pixel) {
    uint64_t z = seed * 0xD1B54A32D192ED03ull + ((uint64_t(frame) << 32) | uint32_t(pixel));
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return uint32_t((z ^ (z >> 31)) >> 32);
}

// Warp-aggregated append returning each taking lane's position (-1 for the others).
__device__ inline int32_t append(bool take, int32_t *counter) {
    unsigned m = __ballot_sync(0xffffffffu, take);
    if (!m) return -1;
    int leader = __ffs(m) - 1;
    int32_t base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    return take ? base + __popc(m & ((1u << lane_id()) - 1u)) : -1;
}

// A fresh camera sample of pixel i (trace_pixel_sample's camera step, transport.h:232-239).
__device__ inline void camera_sample(const Params &p, int32_t i, Pcg &rng, int32_t train, int32_t samples_left, CachePath &s) {
    int x = i % p.width, y = i / p.width;
    float u = (x + rng.uniform()) / float(p.width);
    float v = (y + rng.uniform()) / float(p.height);
    pt_ray r;
    camera_ray(p.camera, u, v, rng, r);
    s.ox = r.origin.x; s.oy = r.origin.y; s.oz = r.origin.z; s.time = r.time;
    s.dx = r.direction.x; s.dy = r.direction.y; s.dz = r.direction.z; s.bounce_pdf = 0;
    s.tr = 1; s.tg = 1; s.tb = 1; s.prev_pdf = 0;
    s.rr = 0; s.rg = 0; s.rb = 0; s.spread = 0;
    s.ur = 1; s.ug = 1; s.ub = 1; s.a0 = 0;
    s.sr = 0; s.sg = 0; s.sb = 0; s.depth = 0;
    s.train = train; s.vertices = -1; s.qdepth = 0; s.samples_left = samples_left;
}

__global__ void start_kernel(Params p, Buffers b, int32_t pixels) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < pixels;
    const uint32_t frame = *b.frame;
    bool train = valid && p.train_threshold && pixel_hash(p.seed, frame, i) < p.train_threshold;
    int32_t slot = append(train, &b.counters[4]);
    if (slot >= p.train_capacity) { train = false; slot = -1; }
    const bool start = valid && (p.accumulate || train);
    if (start) {
        Pcg rng = b.rng[i];
        CachePath s;
        camera_sample(p, i, rng, train ? slot : -1, p.spf, s);   // a training pixel trains on its first sample
        b.rng[i] = rng;
        b.paths[i] = s;
        if (p.accumulate) b.pixel_query_count[i] = 0;
    }
    push(start, i, b.queue[0], &b.counters[0]);
}

// A prediction of L / albedo, bounded by the brightest emitter: with no emitted radiance above
// Le_max, no outgoing radiance exceeds albedo * Le_max (a diffuse, mirror or glass vertex
// passes on at most albedo times its brightest incoming radiance).  A prediction outside
// [0, Le_max] cannot be right; the clamp keeps a badly extrapolated query from becoming a
// firefly.
__device__ inline float bounded(float prediction, float bound) {
    return prediction >= 0.0f ? fminf(prediction, bound) : 0.0f;
}

__device__ inline pt_ray cache_ray(const CachePath &s) {
    pt_ray r;
    r.origin = pt_vec3{s.ox, s.oy, s.oz};
    r.direction = pt_vec3{s.dx, s.dy, s.dz};
    r.time = s.time;
    return r;
}

__global__ void __launch_bounds__(256, 4) extend_kernel(DeviceScene scene, Params p, Buffers b, int parity, int min_active) {
    const int32_t n = b.counters[parity];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&b.totals[0], (unsigned long long)n);
        b.counters[parity ^ 1] = 0;
        b.counters[kShadowSlot + parity] = 0;   // this iteration's shadow slot (the other may be in use)
        b.fetch[1 + parity] = 0;
    }
    const int32_t *queue = b.queue[parity];
    auto get = [&](size_t k, pt_ray &r, float &lo, float &hi) { r = cache_ray(b.paths[queue[k]]); lo = 0.001f; hi = FLT_MAX; };
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
}

struct ShadeOut {
    bool live = false, shadow = false, query = false, finished = false;
    pt_cache_query q;
    QueryAux aux;
    CacheShadow sr;
    f3 tail_weight;
};

// One bounce of path i given its closest hit (see the file comment).
__device__ inline void shade(const DeviceScene &scene, const Params &p, const Buffers &b, int32_t i, CachePath &s,
                             const PathHit &h, Pcg &rng, ShadeOut &o) {
    f3 R = mk(s.rr, s.rg, s.rb), T = mk(s.tr, s.tg, s.tb), U = mk(s.ur, s.ug, s.ub), S = mk(s.sr, s.sg, s.sb);
    o.tail_weight = mk(0, 0, 0);
    if (h.slot < 0) {
        o.finished = true;                          // miss (black background) or a traversal error
    } else {
        pt_ray r = cache_ray(s);
        HitInfo hi; hi.t = h.t; hi.u = h.u; hi.v = h.v; hi.slot = h.slot;
        pt_flat_hit rec;
        finalize_hit(scene, r, hi, rec);
        const pt_material mat = scene.materials[rec.material_id];
        f3 d = mk(s.dx, s.dy, s.dz), pos = mk(rec.p), normal = mk(rec.normal);
        const float dl2 = sqlen(d);
        const float dist2 = h.t * h.t * dl2;
        const float cosine = fmaxf(fabsf(dot(normal, d)) / sqrtf(dl2), 1e-4f);
        if (s.depth == 0) s.a0 = dist2 / (4.0f * float(M_PI) * cosine);
        else if (s.bounce_pdf > 0) s.spread += sqrtf(dist2 / (s.bounce_pdf * cosine));
        const bool suffix = s.vertices >= 0;
        if (mat.type == PT_LIGHT) {
            float weight = s.prev_pdf > 0 ? mis_weight(s.prev_pdf, hit_light_pdf(scene, mk(s.ox, s.oy, s.oz), rec)) : 1;
            f3 e = weight * trace_texture(scene, mat.texture_id, rec.u, rec.v);
            R = R + T * e;
            if (suffix) S = S + U * e;
            o.finished = true;
        } else if (s.depth == p.max_depth) {
            o.finished = true;
        } else {
            const bool diffuse = mat.type == PT_DIFFUSE;
            // The cache answers at diffuse vertices, and with query_specular also at metal and
            // glass ones (roughness = fuzz, 0 for glass; albedo 1 for glass).
            const bool cacheable = diffuse || (p.query_specular && (mat.type == PT_METAL || mat.type == PT_GLASS));
            const f3 albedo = mat.type == PT_GLASS ? mk(1, 1, 1)
                            : mat.type == PT_METAL ? mk(mat.albedo) : trace_texture(scene, mat.texture_id, rec.u, rec.v);
            bool stop = false;
            if (cacheable && p.use_cache) {
                const bool at_query = !suffix && s.depth >= 1 && s.spread * s.spread > p.spread_c * s.a0;
                pt_cache_query cq;
                cq.position = rec.p; cq.direction = pv(-(d / sqrtf(dl2))); cq.normal = rec.normal; cq.albedo = pv(albedo);
                cq.roughness = diffuse ? 1.0f : (mat.type == PT_METAL ? fminf(mat.fuzz, 1.0f) : 0.0f);
                if (at_query && s.train < 0) {
                    stop = true;
                } else if (s.train >= 0) {
                    if (at_query) { s.vertices = 0; s.qdepth = s.depth; }
                    if (s.vertices >= 0) {
                        if (s.depth - s.qdepth >= p.suffix_bounces) {
                            stop = true;
                            o.tail_weight = U * albedo;
                        } else if (s.vertices < p.suffix_bounces) {
                            TrainVertex tv;
                            tv.q = cq;
                            tv.sr = S.x; tv.sg = S.y; tv.sb = S.z;
                            tv.ur = U.x; tv.ug = U.y; tv.ub = U.z; tv.pad = 0;
                            b.vertices[size_t(s.train) * kMaxSuffix + s.vertices] = tv;
                            s.vertices++;
                        }
                    }
                }
                if (stop) {
                    o.q = cq;
                    f3 w = T * albedo;
                    o.aux.wr = w.x; o.aux.wg = w.y; o.aux.wb = w.z; o.aux.path = i;
                    o.query = true;
                    o.finished = true;
                }
            }
            if (stop) {
            } else if (diffuse) {
                const bool in_suffix = s.vertices >= 0;
                if (scene.light_count) {
                    LightSample light = sample_light(scene, rng);
                    f3 delta = light.point - pos;
                    float distance = length(delta);
                    if (distance > 0.002f && finite(distance)) {
                        f3 direction = delta / distance;
                        float cosl = fmaxf(0, dot(normal, direction));
                        float pdf = light_direction_pdf(scene.light_area, pos, light.point, light.normal);
                        if (cosl > 0 && pdf > 0) {
                            const pt_material &emitter = scene.materials[light.material];
                            f3 emission = trace_texture(scene, emitter.texture_id, light.u, light.v);
                            float bsdf_pdf = cosl / float(M_PI);
                            f3 local = albedo * emission * (bsdf_pdf * mis_weight(pdf, bsdf_pdf) / pdf);
                            f3 c = T * local, cs = U * local;
                            CacheShadow &sr = o.sr;
                            sr.ox = pos.x; sr.oy = pos.y; sr.oz = pos.z; sr.tmax = distance - 0.001f;
                            sr.dx = direction.x; sr.dy = direction.y; sr.dz = direction.z; sr.time = s.time;
                            sr.cr = c.x; sr.cg = c.y; sr.cb = c.z; sr.path = i;
                            sr.sr = cs.x; sr.sg = cs.y; sr.sb = cs.z; sr.suffix = in_suffix ? 1 : 0;
                            o.shadow = true;
                        }
                    }
                }
                f3 direction = cosine_direction(normal, rng);
                s.prev_pdf = fmaxf(0, dot(normal, direction)) / float(M_PI);
                s.bounce_pdf = s.prev_pdf;
                T = T * albedo;
                U = U * albedo;
                s.ox = pos.x; s.oy = pos.y; s.oz = pos.z;
                s.dx = direction.x; s.dy = direction.y; s.dz = direction.z;
                s.depth++;
            } else {
                s.prev_pdf = 0;
                s.bounce_pdf = 0;                   // a delta lobe adds no spread
                f3 attenuation, dir;
                if (!trace_scatter(scene, mat, d, rec, rng, attenuation, dir)) o.finished = true;
                else {
                    T = T * attenuation;
                    U = U * attenuation;
                    s.ox = pos.x; s.oy = pos.y; s.oz = pos.z;
                    s.dx = dir.x; s.dy = dir.y; s.dz = dir.z;
                    s.depth++;
                }
            }
        }
    }
    s.tr = T.x; s.tg = T.y; s.tb = T.z;
    s.rr = R.x; s.rg = R.y; s.rb = R.z;
    s.ur = U.x; s.ug = U.y; s.ub = U.z;
    s.sr = S.x; s.sg = S.y; s.sb = S.z;
    o.live = !o.finished;
}

// Book-keeping of a path sample that ended this bounce: its radiance into the pixel sum, its
// cache query (index `q`) into the pixel's query list (the resolve step adds the weighted
// prediction), a training path's end record.  Then the pixel's next sample starts, if any;
// returns whether the path goes on.
__device__ inline bool retire(const Params &p, const Buffers &b, int32_t i, CachePath &s, Pcg &rng, const ShadeOut &o, int32_t q) {
    if (p.accumulate) {
        float *sum = b.sums + 3 * size_t(i);
        sum[0] += s.rr; sum[1] += s.rg; sum[2] += s.rb;
    }
    if (o.query) {
        b.queries[q] = o.q;
        b.aux[q] = o.aux;
        if (p.accumulate) {
            int32_t j = b.pixel_query_count[i];
            b.pixel_queries[size_t(i) * p.spf + j] = q;
            b.pixel_query_count[i] = j + 1;
        }
    }
    if (s.train >= 0) {
        TrainEnd e;
        e.sr = s.sr; e.sg = s.sg; e.sb = s.sb; e.query = o.query ? q : -1;
        e.wr = o.tail_weight.x; e.wg = o.tail_weight.y; e.wb = o.tail_weight.z;
        e.vertices = s.vertices > 0 ? s.vertices : 0;
        b.ends[s.train] = e;
    }
    if (s.samples_left > 1) {
        camera_sample(p, i, rng, -1, s.samples_left - 1, s);
        return true;
    }
    return false;
}

__global__ void shade_kernel(DeviceScene scene, Params p, Buffers b, int parity) {
    const int32_t n = b.counters[parity];
    const int32_t *in = b.queue[parity];
    int32_t *out = b.queue[parity ^ 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) b.fetch[0] = 0;
    for (int32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const int32_t k = base + threadIdx.x;
        const bool valid = k < n;
        const int32_t i = valid ? in[k] : 0;
        ShadeOut o;
        CachePath s;
        Pcg rng;
        if (valid) {
            s = b.paths[i];
            PathHit h = b.hits[i];
            rng = b.rng[i];
            shade(scene, p, b, i, s, h, rng, o);
            if (o.shadow) b.shadows[i] = o.sr;
        }
        const int32_t q = append(o.query, &b.counters[3]);
        bool live = o.live;
        if (valid) {
            if (o.finished) live = retire(p, b, i, s, rng, o, q);
            b.rng[i] = rng;
            b.paths[i] = s;
        }
        push(live, i, out, &b.counters[parity ^ 1]);
        push(o.shadow, i, b.shadow_queue, &b.counters[kShadowSlot + parity]);
    }
}

// finish: the queue's remaining paths run to their end, one thread per path (extend, shade and
// shadow fused).  Runs once the queue is short, where a wavefront iteration would cost the
// latency of its slowest ray for a handful of rays; used on two-wide trees (four-wide trees take
// finish_pair_kernel below).
__global__ void finish_kernel(DeviceScene scene, Params p, Buffers b, int parity) {
    const int32_t n = b.counters[parity];
    unsigned long long rays = 0;
    for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int32_t i = b.queue[parity][k];
        CachePath s = b.paths[i];
        Pcg rng = b.rng[i];
        for (;;) {
            rays++;
            pt_ray r = cache_ray(s);
            HitInfo hi;
            uint32_t boxes = 0, prims = 0;
            int error = 0;
            bool hit = p.wide ? traverse4<false>(scene, r, 0.001f, FLT_MAX, kTieLastLeaf, hi, boxes, prims, error)
                              : traverse<false>(scene, r, 0.001f, FLT_MAX, kTieLastLeaf, hi, boxes, prims, error);
            if (error) *b.error = 1;
            PathHit h;
            h.t = hi.t; h.u = hi.u; h.v = hi.v; h.slot = (hit && !error) ? hi.slot : (error ? -2 : -1);
            ShadeOut o;
            shade(scene, p, b, i, s, h, rng, o);
            if (o.shadow) {
                rays++;
                const CacheShadow &sr = o.sr;
                pt_ray q;
                q.origin = pt_vec3{sr.ox, sr.oy, sr.oz};
                q.direction = pt_vec3{sr.dx, sr.dy, sr.dz};
                q.time = sr.time;
                HitInfo sh;
                uint32_t sb = 0, sp = 0;
                int serr = 0;
                bool blocked = p.wide ? traverse4<true>(scene, q, 0.001f, sr.tmax, kTieLastLeaf, sh, sb, sp, serr)
                                      : traverse<true>(scene, q, 0.001f, sr.tmax, kTieLastLeaf, sh, sb, sp, serr);
                if (serr) *b.error = 1;
                else if (!blocked) {
                    s.rr += sr.cr; s.rg += sr.cg; s.rb += sr.cb;
                    if (sr.suffix) { s.sr += sr.sr; s.sg += sr.sg; s.sb += sr.sb; }
                }
            }
            if (o.finished) {
                const int32_t q = o.query ? atomicAdd(&b.counters[3], 1) : -1;
                if (!retire(p, b, i, s, rng, o, q)) break;
            }
        }
        b.paths[i] = s;
        b.rng[i] = rng;
    }
    for (int o = 16; o; o >>= 1) rays += __shfl_down_sync(0xffffffffu, rays, o);
    if ((threadIdx.x & 31) == 0 && rays) atomicAdd(&b.totals[0], rays);
}

// finish, two lanes per path (four-wide tree): in each round the even lane of a pair walks the
// path's next ray while the odd lane walks the shadow ray of the path's previous bounce, through
// one runtime-mode walk (traverse4_rt), so a bounce costs one walk's latency instead of two.  A
// bounce that emits a shadow ray never ends its path sample, and the shadow contribution of
// bounce k is added before bounce k+1 is shaded (or its sample retired), as in the one-lane
// form.  A pair whose path has ended takes the next queue entry from fetch[3].
__global__ void __launch_bounds__(256, 2) finish_pair_kernel(DeviceScene scene, Params p, Buffers b, int parity) {
    const int32_t n = b.counters[parity];
    const unsigned full = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31;
    const bool odd = lane & 1;
    const unsigned even_lane = lane & ~1u, odd_lane = lane | 1u;
    unsigned long long rays = 0;
    int32_t i = -1;                // even lane: the path (slot) in hand, -1 when none
    CachePath s{};
    Pcg rng{};
    bool live = false;             // even lane: the path has a ray to walk
    bool pending = false;          // even lane: a shadow ray from the last shading waits
    bool drained = false;          // even lane: the queue had no entry left for this pair
    CacheShadow sr{};              // even lane: the pending shadow ray
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
            rays++;
            hit = traverse4_rt(scene, odd ? q : cache_ray(s), 0.001f, odd ? qmax : FLT_MAX, kTieLastLeaf, odd, hi, boxes, prims,
                               error);
        }
        const bool blocked = __shfl_sync(full, hit, odd_lane);
        const int shadow_error = __shfl_sync(full, error, odd_lane);
        if (!odd) {
            if (pending) {
                if (shadow_error) *b.error = 1;
                else if (!blocked) {
                    s.rr += sr.cr; s.rg += sr.cg; s.rb += sr.cb;
                    if (sr.suffix) { s.sr += sr.sr; s.sg += sr.sg; s.sb += sr.sb; }
                }
                pending = false;
            }
            if (live) {
                if (error) *b.error = 1;
                PathHit h;
                h.t = hi.t; h.u = hi.u; h.v = hi.v; h.slot = (hit && !error) ? hi.slot : (error ? -2 : -1);
                ShadeOut o;
                shade(scene, p, b, i, s, h, rng, o);
                if (o.shadow) { sr = o.sr; pending = true; }
                if (o.finished) {
                    const int32_t qi = o.query ? atomicAdd(&b.counters[3], 1) : -1;
                    live = retire(p, b, i, s, rng, o, qi);
                }
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
    if (lane == 0 && rays) atomicAdd(&b.totals[0], rays);
}

__global__ void __launch_bounds__(256, 4) shadow_kernel(DeviceScene scene, Params p, Buffers b, int parity, int min_active) {
    const int32_t n = b.counters[kShadowSlot + parity];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&b.totals[0], (unsigned long long)n);
    auto get = [&](size_t k, pt_ray &r, float &lo, float &hi) {
        const CacheShadow &sr = b.shadows[b.shadow_queue[k]];
        r.origin = pt_vec3{sr.ox, sr.oy, sr.oz};
        r.direction = pt_vec3{sr.dx, sr.dy, sr.dz};
        r.time = sr.time;
        lo = 0.001f; hi = sr.tmax;
    };
    auto done = [&](size_t k, const WalkResult &w) {
        if (w.error) { *b.error = 1; return; }
        if (w.slot >= 0) return;
        const int32_t i = b.shadow_queue[k];
        const CacheShadow sr = b.shadows[i];
        CachePath &s = b.paths[i];
        s.rr += sr.cr; s.rg += sr.cg; s.rb += sr.cb;
        if (sr.suffix) { s.sr += sr.sr; s.sg += sr.sg; s.sb += sr.sb; }
    };
    if (p.wide == 2) persistent_walk4_spec<true>(scene, size_t(n), &b.fetch[1 + parity], min_active, kTieLastLeaf, get, done);
    else if (p.wide) persistent_walk4<true>(scene, size_t(n), &b.fetch[1 + parity], min_active, kTieLastLeaf, get, done);
    else persistent_walk<true>(scene, size_t(n), &b.fetch[1 + parity], min_active, kTieLastLeaf, get, done);
}

// Pixel sums += weight x prediction of the pixel's queries, in sample order.
__global__ void resolve_kernel(Params p, Buffers b, int32_t pixels) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&b.totals[1], (unsigned long long)b.counters[3]);
    if (!p.accumulate) return;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pixels; i += gridDim.x * blockDim.x) {
        const int32_t n = b.pixel_query_count[i];
        if (!n) continue;
        float *sum = b.sums + 3 * size_t(i);
        float acc[3] = {sum[0], sum[1], sum[2]};
        for (int32_t j = 0; j < n; j++) {
            const int32_t q = b.pixel_queries[size_t(i) * p.spf + j];
            const QueryAux a = b.aux[q];
            acc[0] += a.wr * bounded(b.pred[3 * size_t(q)], p.radiance_max[0]);
            acc[1] += a.wg * bounded(b.pred[3 * size_t(q) + 1], p.radiance_max[1]);
            acc[2] += a.wb * bounded(b.pred[3 * size_t(q) + 2], p.radiance_max[2]);
        }
        sum[0] = acc[0]; sum[1] = acc[1]; sum[2] = acc[2];
    }
}

// Training samples of the frame's training paths (see the file comment).
__global__ void targets_kernel(Params p, Buffers b) {
    const int32_t n = min(b.counters[4], p.train_capacity);
    for (int32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const TrainEnd e = b.ends[t];
        float total[3] = {e.sr, e.sg, e.sb};
        if (e.query >= 0) {
            total[0] += e.wr * bounded(b.pred[3 * size_t(e.query)], p.radiance_max[0]);
            total[1] += e.wg * bounded(b.pred[3 * size_t(e.query) + 1], p.radiance_max[1]);
            total[2] += e.wb * bounded(b.pred[3 * size_t(e.query) + 2], p.radiance_max[2]);
        }
        const int bucket = t % p.steps;
        for (int v = 0; v < e.vertices && v < kMaxSuffix; v++) {
            const TrainVertex tv = b.vertices[size_t(t) * kMaxSuffix + v];
            const float s[3] = {tv.sr, tv.sg, tv.sb}, u[3] = {tv.ur, tv.ug, tv.ub};
            const float a[3] = {tv.q.albedo.x, tv.q.albedo.y, tv.q.albedo.z};
            float target[3];
            bool ok = true;
            for (int c = 0; c < 3; c++) {
                float den = u[c] * a[c];
                float value = fmaxf(total[c] - s[c], 0.0f) / den;
                ok = ok && den > 1e-12f && finite(value);
                target[c] = value;
            }
            if (!ok) continue;
            const int32_t idx = atomicAdd(&b.counters[5 + bucket], 1);
            if (idx >= p.bucket_capacity) continue;
            const size_t at = size_t(bucket) * size_t(p.bucket_capacity) + size_t(idx);
            b.samples[at] = tv.q;
            b.targets[3 * at] = target[0]; b.targets[3 * at + 1] = target[1]; b.targets[3 * at + 2] = target[2];
        }
    }
}

__global__ void frame_end_kernel(Params p, Buffers b) {
    if (threadIdx.x != 0) return;
    unsigned long long samples = 0;
    for (int s = 0; s < p.steps; s++) samples += (unsigned long long)min(b.counters[5 + s], p.bucket_capacity);
    b.totals[2] += samples;
    b.frame[0] += 1;
}

// One thread: go on with the WHILE loop while at least tail_paths paths are live (the fused
// kernel ends a shorter tail); past the iteration bound the frame stops with an error.
__global__ void control_kernel(Buffers b, cudaGraphConditionalHandle handle, int32_t tail_paths, unsigned long long max_pairs) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int32_t live = b.counters[0];
    const unsigned long long pair = ++*b.pairs;
    bool go = live > 0 && live >= tail_paths;
    if (go && pair >= max_pairs) { *b.error = 2; go = false; }
    cudaGraphSetConditional(handle, go ? 1u : 0u);
}

} // namespace nrc
} // namespace ptb

using namespace ptb::nrc;

struct pt_cached_renderer {
    const pt_scene *scene = nullptr;
    pt_cache *cache = nullptr;
    pt_cached_params cfg{};
    Params params{};
    int32_t pixels = 0;
    int frames = 0;
    float milliseconds = 0;
    int block = 256;
    int grid_extend = 0, grid_shade = 0, grid_shadow = 0, grid_finish = 0, grid_finish_pair = 0, grid_small = 0;
    DeviceBuffer paths, hits, shadows, queue0, queue1, shadow_queue, counters, fetch, totals, error, sums, rng, frame;
    DeviceBuffer queries, aux, pred, pixel_queries, pixel_query_count, vertices, ends, samples, targets;
    Buffers buf{};
    cudaStream_t stream = nullptr, body_stream = nullptr, shadow_stream = nullptr;
    Event shaded[2], shadowed[2];
    Event start, stop;
    int32_t tail_paths = 0;             // live paths below which the fused kernel ends the frame
    int32_t *live_host = nullptr;       // pinned: live count read back by the launched form
    DeviceBuffer pairs;
    bool training = true;               // online training on (pt_cached_training)
    cudaGraphExec_t exec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [accumulate][training]
    ~pt_cached_renderer() {
        for (auto &row : exec) for (auto &e : row) if (e) cudaGraphExecDestroy(e);
        if (cache) pt_cache_destroy(cache);
        if (live_host) cudaFreeHost(live_host);
        if (body_stream) cudaStreamDestroy(body_stream);
        if (shadow_stream) cudaStreamDestroy(shadow_stream);
        if (stream) cudaStreamDestroy(stream);
    }
    // the launches of one frame (also what a graph captures)
    Params frame_params(int accumulate) const {
        Params p = params;
        p.accumulate = accumulate;
        if (!accumulate) p.spf = 1;                 // training-only frames: the training sample alone
        if (!training) p.train_threshold = 0;       // no training paths: every pixel may end at the cache
        return p;
    }
    // A pixel's samples run one after another: at most spf * (max_depth + 1) bounces, so the
    // wavefront ends within that many iterations (the pair loop's bound, with a margin).
    unsigned long long max_pairs(const Params &p) const {
        return (unsigned long long)p.spf * (unsigned long long)(p.max_depth + 1) / 2 + 2;
    }
    void prologue(const Params &p, cudaStream_t st) {
        PT_CUDA(cudaMemsetAsync(buf.counters, 0, kCounters * sizeof(int32_t), st));
        PT_CUDA(cudaMemsetAsync(buf.fetch, 0, 4 * sizeof(unsigned long long), st));
        PT_CUDA(cudaMemsetAsync(buf.pairs, 0, sizeof(unsigned long long), st));
        start_kernel<<<(pixels + 255) / 256, 256, 0, st>>>(p, buf, pixels);
        PT_CUDA(cudaGetLastError());
    }
    // Two iterations.  The first one's shadow kernel runs on the shadow stream beside the
    // second one's extend; shade waits for the shadow kernel before it (it rewrites the shadow
    // records and reads the radiance the shadow kernel adds); the pair ends joined.
    void iteration_pair(const Params &p, cudaStream_t st) {
        for (int parity = 0; parity < 2; parity++) {
            extend_kernel<<<grid_extend, block, stack_bytes(block), st>>>(scene->view, p, buf, parity, g_query_config.min_active);
            if (parity == 1) PT_CUDA(cudaStreamWaitEvent(st, shadowed[0].get(), 0));
            shade_kernel<<<grid_shade, block, 0, st>>>(scene->view, p, buf, parity);
            PT_CUDA(cudaEventRecord(shaded[parity].get(), st));
            PT_CUDA(cudaStreamWaitEvent(shadow_stream, shaded[parity].get(), 0));
            shadow_kernel<<<grid_shadow, block, stack_bytes(block), shadow_stream>>>(scene->view, p, buf, parity,
                                                                                    g_query_config.min_active);
            PT_CUDA(cudaEventRecord(shadowed[parity].get(), shadow_stream));
        }
        PT_CUDA(cudaStreamWaitEvent(st, shadowed[1].get(), 0));
        PT_CUDA(cudaGetLastError());
    }
    // the fused kernel ends the paths left in queue 0, then the network's part of the frame
    void epilogue(const Params &p, cudaStream_t st) {
        if (p.wide) finish_pair_kernel<<<grid_finish_pair, block, 0, st>>>(scene->view, p, buf, 0);
        else finish_kernel<<<grid_finish, block, 0, st>>>(scene->view, p, buf, 0);
        PT_CUDA(cudaGetLastError());
        if (p.use_cache) {
            cache_forward(cache, buf.queries, query_capacity(), &buf.counters[3], buf.pred, st);
            resolve_kernel<<<grid_small, 256, 0, st>>>(p, buf, pixels);
            PT_CUDA(cudaGetLastError());
            if (p.train_threshold) {
                targets_kernel<<<grid_small, 256, 0, st>>>(p, buf);
                PT_CUDA(cudaGetLastError());
                for (int s = 0; s < p.steps; s++) {
                    size_t at = size_t(s) * size_t(p.bucket_capacity);
                    cache_train(cache, buf.samples + at, buf.targets + 3 * at, size_t(p.bucket_capacity), &buf.counters[5 + s], st);
                }
            }
        }
        frame_end_kernel<<<1, 32, 0, st>>>(p, buf);
        PT_CUDA(cudaGetLastError());
    }
    // One frame launched kernel by kernel: wavefront iteration pairs while at least tail_paths
    // paths are live (the live count read back after each pair), then the epilogue.
    void launch_frame(int accumulate) {
        const Params p = frame_params(accumulate);
        cudaStream_t st = stream;
        prologue(p, st);
        const unsigned long long bound = max_pairs(p);
        for (unsigned long long pair = 0;; pair++) {
            iteration_pair(p, st);
            PT_CUDA(cudaMemcpyAsync(live_host, &buf.counters[0], sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            PT_CUDA(cudaStreamSynchronize(st));
            if (*live_host < tail_paths) break;
            if (pair + 1 >= bound) throw Error(PT_TIMEOUT, "wavefront did not drain within its iteration bound");
        }
        epilogue(p, st);
    }
    // The same frame as one graph: prologue, a WHILE node whose body is an iteration pair and
    // the control kernel (the device decides when the tail is short), epilogue.
    void capture_frame(int accumulate, cudaGraph_t *out) {
        const Params p = frame_params(accumulate);
        PT_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
            prologue(p, stream);
            cudaStreamCaptureStatus status;
            cudaGraph_t g = nullptr;
            const cudaGraphNode_t *deps = nullptr;
            size_t ndeps = 0;
            PT_CUDA(cudaStreamGetCaptureInfo(stream, &status, nullptr, &g, &deps, &ndeps));
            cudaGraphConditionalHandle handle;
            PT_CUDA(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams cp{};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = handle;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t loop;
            PT_CUDA(cudaGraphAddNode(&loop, g, deps, ndeps, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            PT_CUDA(cudaStreamBeginCaptureToGraph(body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
            iteration_pair(p, body_stream);
            control_kernel<<<1, 32, 0, body_stream>>>(buf, handle, tail_paths, max_pairs(p));
            PT_CUDA(cudaGetLastError());
            PT_CUDA(cudaStreamEndCapture(body_stream, &body));
            PT_CUDA(cudaStreamUpdateCaptureDependencies(stream, &loop, 1, cudaStreamSetCaptureDependencies));
            epilogue(p, stream);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        PT_CUDA(cudaStreamEndCapture(stream, out));
    }
    size_t query_capacity() const { return size_t(pixels) * size_t(params.spf); }
    cudaGraphExec_t graph(int accumulate) {
        cudaGraphExec_t &slot = exec[accumulate][training ? 1 : 0];
        if (slot) return slot;
        cudaGraph_t g = nullptr;
        capture_frame(accumulate, &g);
        cudaError_t e = cudaGraphInstantiate(&slot, g, 0);
        cudaGraphDestroy(g);
        PT_CUDA(e);
        return slot;
    }
};

namespace {
void defaults(pt_cached_params &c) {
    c.training_paths = 65536; c.train_steps = 1; c.suffix_bounces = 4; c.use_cache = 1; c.train = 1; c.use_graph = 1;
    c.spread_threshold = 0.3f; c.learning_rate = 1e-2f; c.network_seed = 7; c.tail_paths = 0;
    c.query_specular = 1; c.weight_average = 0.99f; c.samples_per_frame = 4;
}
} // namespace

extern "C" {

pt_status pt_cached_defaults(pt_cached_params *params) {
    return guard([&]() {
        if (!params) throw Error(PT_INVALID_ARGUMENT, "null argument");
        defaults(*params);
    });
}

pt_status pt_cached_create(const pt_scene *scene, const pt_camera *camera, int width, int height, uint64_t seed, int max_depth,
                           const pt_cached_params *params, pt_cached_renderer **out) {
    return guard([&]() {
        if (!scene || !camera || !out) throw Error(PT_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        pt_cached_params cfg;
        if (params) cfg = *params; else defaults(cfg);
        if (width <= 0 || height <= 0 || uint64_t(width) * uint64_t(height) > uint64_t(INT32_MAX / 4))
            throw Error(PT_INVALID_ARGUMENT, "image dimensions exceed supported pixel count");
        if (max_depth < 0 || max_depth > 1000) throw Error(PT_INVALID_ARGUMENT, "invalid bounce limit");
        if (cfg.training_paths < 0 || cfg.train_steps < 1 || cfg.train_steps > kMaxSteps || cfg.suffix_bounces < 1 ||
            cfg.suffix_bounces > kMaxSuffix || !(cfg.spread_threshold >= 0) || !(cfg.learning_rate > 0) ||
            cfg.tail_paths < 0 || !(cfg.weight_average >= 0 && cfg.weight_average < 1) ||
            cfg.samples_per_frame < 1 || cfg.samples_per_frame > 64)
            throw Error(PT_INVALID_ARGUMENT, "invalid radiance-cache settings");
        for (const pt_vec3 &v : {camera->origin, camera->lower_left_corner, camera->horizontal, camera->vertical})
            if (!std::isfinite(v.x) || !std::isfinite(v.y) || !std::isfinite(v.z))
                throw Error(PT_INVALID_ARGUMENT, "camera contains nonfinite values");
        require_device();
        auto r = new pt_cached_renderer;
        try {
            const size_t n = size_t(width) * size_t(height);
            r->scene = scene;
            r->cfg = cfg;
            r->pixels = int32_t(n);
            float lo[3], hi[3];
            for (int a = 0; a < 3; a++) { lo[a] = scene->view.root_lo[a]; hi[a] = scene->view.root_hi[a]; }
            if (!(hi[0] > lo[0]) || !(hi[1] > lo[1]) || !(hi[2] > lo[2])) {   // empty or flat scene: a unit box
                for (int a = 0; a < 3; a++) { if (!std::isfinite(lo[a])) lo[a] = 0; hi[a] = std::max(hi[a], lo[a] + 1.0f); }
            }
            pt_status st = pt_cache_create(lo, hi, cfg.network_seed, &r->cache);
            if (st != PT_OK) throw Error(st, pt_last_error());
            st = pt_cache_hyper(r->cache, cfg.learning_rate, 0.9f, 0.99f, 1e-8f);
            if (st != PT_OK) throw Error(st, pt_last_error());
            st = pt_cache_average(r->cache, cfg.weight_average);
            if (st != PT_OK) throw Error(st, pt_last_error());
            const bool training = cfg.use_cache && cfg.train && cfg.training_paths > 0;
            const int32_t capacity = training ? int32_t(std::min<int64_t>(int64_t(n), int64_t(cfg.training_paths) * 5 / 4 + 1024)) : 0;
            Params &p = r->params;
            p.camera = *camera; p.width = width; p.height = height; p.max_depth = max_depth;
            p.wide = (g_query_config.wide && scene->view.nodes4) ? (g_query_config.speculative ? 2 : 1) : 0;
            p.use_cache = cfg.use_cache ? 1 : 0;
            p.suffix_bounces = cfg.suffix_bounces;
            p.query_specular = cfg.query_specular ? 1 : 0;
            p.spf = cfg.samples_per_frame;
            p.steps = cfg.train_steps;
            p.spread_c = cfg.spread_threshold;
            p.seed = seed;
            double fraction = training ? std::min(1.0, double(cfg.training_paths) / double(n)) : 0.0;
            p.train_threshold = training ? uint32_t(std::min(4294967295.0, std::ceil(fraction * 4294967296.0))) : 0u;
            p.train_capacity = capacity;
            p.bucket_capacity = training ? (capacity + p.steps - 1) / p.steps * p.suffix_bounces : 0;
            {
                // brightest emitted radiance: constant colour, image texel (<= 1) or colour x texel
                std::vector<pt_material> mats(scene->materials.bytes() / sizeof(pt_material));
                std::vector<pt_texture> texs(scene->textures.bytes() / sizeof(pt_texture));
                if (!mats.empty()) PT_CUDA(cudaMemcpy(mats.data(), scene->materials.get(), mats.size() * sizeof(pt_material), cudaMemcpyDeviceToHost));
                if (!texs.empty()) PT_CUDA(cudaMemcpy(texs.data(), scene->textures.get(), texs.size() * sizeof(pt_texture), cudaMemcpyDeviceToHost));
                float bound[3] = {0, 0, 0};
                for (const pt_material &m : mats) {
                    if (m.type != PT_LIGHT || m.texture_id < 0 || size_t(m.texture_id) >= texs.size()) continue;
                    const pt_texture &t = texs[size_t(m.texture_id)];
                    const float c[3] = {t.color.x, t.color.y, t.color.z};
                    for (int a = 0; a < 3; a++) bound[a] = std::max(bound[a], t.type == PT_TEX_IMAGE ? 1.0f : std::fabs(c[a]));
                }
                for (int a = 0; a < 3; a++) p.radiance_max[a] = bound[a];
            }
            r->paths.resize(n * sizeof(CachePath));
            r->hits.resize(n * sizeof(PathHit));
            r->shadows.resize(n * sizeof(CacheShadow));
            r->queue0.resize(n * sizeof(int32_t));
            r->queue1.resize(n * sizeof(int32_t));
            r->shadow_queue.resize(n * sizeof(int32_t));
            r->counters.resize(kCounters * sizeof(int32_t));
            r->fetch.resize(4 * sizeof(unsigned long long));
            r->totals.resize(3 * sizeof(unsigned long long));
            r->error.resize(sizeof(int32_t));
            r->sums.resize(n * 3 * sizeof(float));
            r->rng.resize(n * sizeof(Pcg));
            r->frame.resize(sizeof(uint32_t));
            r->pixel_query_count.resize(n * sizeof(int32_t));
            if (cfg.use_cache) {
                const size_t nq = n * size_t(cfg.samples_per_frame);   // at most one query per sample
                r->queries.resize(nq * sizeof(pt_cache_query));
                r->aux.resize(nq * sizeof(QueryAux));
                r->pred.resize(nq * 3 * sizeof(float));
                r->pixel_queries.resize(nq * sizeof(int32_t));
            }
            if (training) {
                r->vertices.resize(size_t(capacity) * kMaxSuffix * sizeof(TrainVertex));
                r->ends.resize(size_t(capacity) * sizeof(TrainEnd));
                size_t total = size_t(p.bucket_capacity) * size_t(p.steps);
                r->samples.resize(total * sizeof(pt_cache_query));
                r->targets.resize(total * 3 * sizeof(float));
            }
            Buffers &b = r->buf;
            b.paths = r->paths.get<CachePath>(); b.hits = r->hits.get<PathHit>(); b.shadows = r->shadows.get<CacheShadow>();
            b.queue[0] = r->queue0.get<int32_t>(); b.queue[1] = r->queue1.get<int32_t>();
            b.shadow_queue = r->shadow_queue.get<int32_t>(); b.counters = r->counters.get<int32_t>();
            b.fetch = r->fetch.get<unsigned long long>(); b.totals = r->totals.get<unsigned long long>();
            b.error = r->error.get<int32_t>(); b.sums = r->sums.get<float>(); b.rng = r->rng.get<Pcg>();
            b.frame = r->frame.get<uint32_t>();
            b.queries = r->queries.get<pt_cache_query>(); b.aux = r->aux.get<QueryAux>(); b.pred = r->pred.get<float>();
            b.pixel_queries = r->pixel_queries.get<int32_t>(); b.pixel_query_count = r->pixel_query_count.get<int32_t>();
            b.vertices = r->vertices.get<TrainVertex>(); b.ends = r->ends.get<TrainEnd>();
            b.samples = r->samples.get<pt_cache_query>(); b.targets = r->targets.get<float>();
            PT_CUDA(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
            PT_CUDA(cudaStreamCreateWithFlags(&r->body_stream, cudaStreamNonBlocking));
            PT_CUDA(cudaStreamCreateWithFlags(&r->shadow_stream, cudaStreamNonBlocking));
            PT_CUDA(cudaMallocHost(&r->live_host, sizeof(int32_t)));
            r->pairs.resize(sizeof(unsigned long long));
            b.pairs = r->pairs.get<unsigned long long>();
            r->tail_paths = cfg.tail_paths > 0 ? cfg.tail_paths : std::max<int32_t>(16384, int32_t(n / 16));
            r->grid_extend = occupancy_grid((const void *)extend_kernel, r->block, stack_bytes(r->block));
            r->grid_shade = occupancy_grid((const void *)shade_kernel, r->block, 0);
            r->grid_shadow = occupancy_grid((const void *)shadow_kernel, r->block, stack_bytes(r->block));
            r->grid_finish = occupancy_grid((const void *)finish_kernel, r->block, 0);
            r->grid_finish_pair = occupancy_grid((const void *)finish_pair_kernel, r->block, 0);
            r->grid_small = device_sm_count() * 4;
            // pixel RNG streams as the plain renderer seeds them (pixel_rng.seed(seed, pixel))
            std::vector<Pcg> streams(n);
            for (size_t i = 0; i < n; i++) streams[i].seed(seed, uint64_t(i));
            PT_CUDA(cudaMemcpy(b.rng, streams.data(), n * sizeof(Pcg), cudaMemcpyHostToDevice));
            PT_CUDA(cudaMemset(b.sums, 0, n * 3 * sizeof(float)));
            PT_CUDA(cudaMemset(b.totals, 0, 3 * sizeof(unsigned long long)));
            PT_CUDA(cudaMemset(b.error, 0, sizeof(int32_t)));
            PT_CUDA(cudaMemset(b.frame, 0, sizeof(uint32_t)));
            PT_CUDA(cudaDeviceSynchronize());
        } catch (...) { delete r; throw; }
        *out = r;
    });
}

pt_status pt_cached_destroy(pt_cached_renderer *r) { delete r; return PT_OK; }

pt_status pt_cached_frames(pt_cached_renderer *r, int frames, int accumulate) {
    return guard([&]() {
        if (!r || frames <= 0 || (accumulate != 0 && accumulate != 1)) throw Error(PT_INVALID_ARGUMENT, "invalid frame request");
        if (accumulate && int64_t(frames) * r->params.spf > int64_t(INT32_MAX - r->frames))
            throw Error(PT_INVALID_ARGUMENT, "invalid accumulated sample count");
        if (!accumulate && !(r->params.train_threshold && r->training))
            throw Error(PT_INVALID_ARGUMENT, "training-only frames need online training");
        cudaGraphExec_t g = r->cfg.use_graph ? r->graph(accumulate) : nullptr;
        PT_CUDA(cudaEventRecord(r->start.get(), r->stream));
        for (int f = 0; f < frames; f++) {
            if (g) PT_CUDA(cudaGraphLaunch(g, r->stream));
            else r->launch_frame(accumulate);
        }
        PT_CUDA(cudaEventRecord(r->stop.get(), r->stream));
        PT_CUDA(cudaEventSynchronize(r->stop.get()));
        int32_t error = 0;
        PT_CUDA(cudaMemcpy(&error, r->buf.error, sizeof error, cudaMemcpyDeviceToHost));
        if (error == 2) throw Error(PT_TIMEOUT, "wavefront did not drain within its iteration bound");
        if (error) throw Error(PT_STACK_OVERFLOW, "CUDA traversal stack overflow");
        cache_status(r->cache);
        float ms = 0;
        PT_CUDA(cudaEventElapsedTime(&ms, r->start.get(), r->stop.get()));
        r->milliseconds += ms;
        if (accumulate) r->frames += frames * r->params.spf;
    });
}

pt_status pt_cached_training(pt_cached_renderer *r, int on) {
    return guard([&]() {
        if (!r || (on != 0 && on != 1)) throw Error(PT_INVALID_ARGUMENT, "invalid training switch");
        r->training = on == 1;
    });
}

pt_status pt_cached_clear(pt_cached_renderer *r) {
    return guard([&]() {
        if (!r) throw Error(PT_INVALID_ARGUMENT, "null renderer");
        PT_CUDA(cudaMemsetAsync(r->buf.sums, 0, size_t(r->pixels) * 3 * sizeof(float), r->stream));
        PT_CUDA(cudaStreamSynchronize(r->stream));
        r->frames = 0;
    });
}

pt_status pt_cached_get_sums(const pt_cached_renderer *r, float *rgb, size_t floats) {
    return guard([&]() {
        if (!r || !rgb || floats < size_t(r->pixels) * 3) throw Error(PT_INVALID_ARGUMENT, "sum buffer too small");
        PT_CUDA(cudaStreamSynchronize(r->stream));
        PT_CUDA(cudaMemcpy(rgb, r->buf.sums, size_t(r->pixels) * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

pt_status pt_cached_stats(pt_cached_renderer *r, int *frames, float *kernel_ms, uint64_t *rays, uint64_t *queries,
                          uint64_t *samples, float *loss) {
    return guard([&]() {
        if (!r) throw Error(PT_INVALID_ARGUMENT, "null renderer");
        unsigned long long t[3] = {0, 0, 0};
        PT_CUDA(cudaStreamSynchronize(r->stream));
        PT_CUDA(cudaMemcpy(t, r->buf.totals, sizeof t, cudaMemcpyDeviceToHost));
        if (frames) *frames = r->frames;
        if (kernel_ms) *kernel_ms = r->milliseconds;
        if (rays) *rays = t[0];
        if (queries) *queries = t[1];
        if (samples) *samples = t[2];
        if (loss) *loss = cache_loss(r->cache, r->stream);
    });
}

pt_status pt_cached_cache(pt_cached_renderer *r, pt_cache **cache) {
    return guard([&]() {
        if (!r || !cache) throw Error(PT_INVALID_ARGUMENT, "null argument");
        *cache = r->cache;
    });
}

} // extern "C"
