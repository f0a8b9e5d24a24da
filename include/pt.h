/*
 * pt.h — C ABI of the B200 path-tracing core.
 *
 * Drop-in boundary for the reference renderer surface of
 * AdmiralHeathCL/cuda-path-tracer:
 *   - `cuda_device_available`           src/cuda/cuda_renderer.h:8
 *   - `class cuda_renderer`             src/cuda/cuda_renderer.h:10-29
 *   - `cuda_query_rays`                 src/cuda/cuda_renderer.h:32
 *   - the flat transfer records         src/flat/flat_data.h:10-62
 *   - `ray`                             src/core/ray.h:6-33
 *   - `trace_result`                    src/renderer/transport.h:12
 *
 * Every record below has the byte layout of the reference record it names,
 * so `flat_scene` vectors can be handed over with `.data()` / `.size()`.
 * No function allocates on behalf of the caller except the opaque handles
 * it returns; every handle owns its device memory and is released by the
 * matching destroy call.  Functions return a pt_status; the message of the
 * last failure on the calling thread is available from pt_last_error().
 */
#ifndef PT_B200_H
#define PT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PT_ABI_VERSION 1

/* ---- status codes (the C++ wrapper maps them to the reference's exception types) ---- */
typedef enum pt_status {
    PT_OK = 0,
    PT_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference (bad dims, sample counts, block shapes) */
    PT_INVALID_SCENE = 2,    /* std::runtime_error("invalid flat scene data"), src/flat/flat_validate.h:12 */
    PT_CUDA_ERROR = 3,       /* std::runtime_error from a failing CUDA call, src/cuda/cuda_renderer.cu:8-11 */
    PT_STACK_OVERFLOW = 4,   /* "CUDA traversal stack overflow", src/cuda/cuda_renderer.cu:204.  trace_world's
                              * stack holds 64 entries and validate_flat_scene bounds a tree's depth at 64,
                              * which keeps it from overflowing (a level leaves at most one entry behind);
                              * this library's walks keep at most 63 (two-wide) or 3 per four-wide level
                              * (192 entries), so a scene pt_scene_create accepts never reports it either */
    PT_QUEUE_OVERFLOW = 5,   /* a wavefront queue would exceed its capacity */
    PT_TIMEOUT = 6,          /* a bounded device-side wait ran out */
    PT_NO_DEVICE = 7         /* cuda_device_available() == false; the CLI exits 77 */
} pt_status;

/* ---- enums, same values as src/flat/flat_data.h:10-12 and src/renderer/transport.h:10 ---- */
enum { PT_BRANCH = 0, PT_TRIANGLE = 1, PT_SPHERE = 2 };
enum { PT_DIFFUSE = 0, PT_METAL = 1, PT_GLASS = 2, PT_LIGHT = 3 };
enum { PT_TEX_CONSTANT = 0, PT_TEX_IMAGE = 1, PT_TEX_MAP = 2 };
enum { PT_DEBUG_SHADED = 0, PT_DEBUG_NORMALS = 1, PT_DEBUG_TRIANGLE = 2, PT_DEBUG_MATERIAL = 3,
       PT_DEBUG_BVH = 4, PT_DEBUG_INTERSECTIONS = 5 };

/* ---- transfer records (byte-compatible with the reference) ---- */
typedef struct pt_vec3 { float x, y, z; } pt_vec3;                       /* vec3, src/core/vec3.h:9 */
typedef struct pt_triangle {                                              /* flat_triangle, 116 B */
    pt_vec3 v0, v1, v2, n0, n1, n2, uv0, uv1, uv2;
    int32_t material_id, smooth;
} pt_triangle;
typedef struct pt_sphere { pt_vec3 center; float radius; int32_t material_id; } pt_sphere; /* flat_sphere, 20 B */
typedef struct pt_node {                                                  /* flat_node, 40 B */
    pt_vec3 minimum, maximum;
    int32_t type, left, right, primitive;
} pt_node;
typedef struct pt_material { pt_vec3 albedo; float fuzz, ref_idx; int32_t type, texture_id; } pt_material; /* 28 B */
typedef struct pt_texture {                                               /* flat_texture, 60 B */
    pt_vec3 color, scale, offset;
    int32_t type, image_id, width, height, byte_offset, clamp;
} pt_texture;
typedef struct pt_camera {                                                /* flat_camera, 84 B */
    pt_vec3 origin, lower_left_corner, horizontal, vertical, u, v;
    float lens_radius, time0, time1;
} pt_camera;
typedef struct pt_ray { pt_vec3 origin, direction; float time; } pt_ray;  /* ray, 28 B */
typedef struct pt_flat_hit {                                              /* flat_hit, 48 B */
    float t, u, v;
    pt_vec3 p, normal;
    int32_t material_id, primitive_type, primitive_id;
} pt_flat_hit;
typedef struct pt_trace_result { pt_flat_hit rec; int32_t hit, error; } pt_trace_result; /* trace_result, 56 B */
typedef struct pt_light { int32_t type, primitive; float cumulative_area; } pt_light;     /* flat_light, 12 B */

/* Compact per-ray answer of pt_query_rays (16 B, one vector store per ray).
 * primitive_type is PT_BRANCH (0) on a miss.  For any-hit queries t is the
 * distance of the first occluder found (not necessarily the closest). */
typedef struct pt_hit { float t; int32_t primitive_id; int32_t primitive_type; int32_t error; } pt_hit;
/* Per-ray traversal counters: child boxes tested and primitives tested. */
typedef struct pt_ray_stats { uint32_t boxes, primitives; } pt_ray_stats;

/* Scene input: the arrays of a reference `flat_scene` (src/flat/flat_data.h:53-62). */
typedef struct pt_scene_desc {
    const pt_triangle *triangles; size_t triangle_count;
    const pt_sphere *spheres;     size_t sphere_count;
    const pt_node *nodes;         size_t node_count;
    const pt_material *materials; size_t material_count;
    const pt_texture *textures;   size_t texture_count;
    const unsigned char *pixels;  size_t pixel_bytes;
    int32_t root;                 /* -1 for an empty scene */
    int32_t max_depth;            /* depth of the tree, root = 1; checked like validate_flat_scene */
} pt_scene_desc;

typedef struct pt_scene pt_scene;       /* device-resident scene (BVH re-laid out, lights table) */
typedef struct pt_renderer pt_renderer; /* progressive renderer state (sums, PCG states, queues) */

/* ---- device probe ----
 * Replaces bool cuda_device_available(std::string&), src/cuda/cuda_renderer.cu:128-140.
 * Writes the device name (or the reason it is unavailable) into `description`. */
int pt_device_available(char *description, size_t capacity);
const char *pt_last_error(void);
int pt_abi_version(void);

/* ---- scene ----
 * Replaces the device_scene upload inside cuda_renderer/cuda_query_rays
 * (src/cuda/cuda_renderer.cu:36-54, 177-183, 248-260): validates with the rules of
 * validate_flat_scene (src/flat/flat_validate.h:10-83), builds the emitter table
 * (scene_lights, src/renderer/scene_view.h:10-28), re-lays the BVH out as 64-byte
 * two-child nodes and the triangles as 48-byte {v0, e1, e2} records, and uploads.
 * The caller's arrays may be freed once this returns. */
pt_status pt_scene_create(const pt_scene_desc *desc, pt_scene **out);
pt_status pt_scene_destroy(pt_scene *scene);
/* Emitter table as built on the host (count, then up to `capacity` records). */
pt_status pt_scene_lights(const pt_scene *scene, pt_light *lights, size_t capacity, size_t *count, float *total_area);
/* Device bytes held by the scene (nodes, triangles, shading records, lights). */
pt_status pt_scene_device_bytes(const pt_scene *scene, size_t *bytes);
/* Host-side check of the four-wide tree pt_scene_create would build for `desc` (no device needed):
 * *nodes = its node count (0 when the scene keeps the two-wide layout), *violations = child
 * bounds whose 8-bit quantised form does not contain the float bounds, plus empty slots that are
 * not inverted (0 for a correct build). */
pt_status pt_layout_check(const pt_scene_desc *desc, size_t *nodes, size_t *violations);
/* Whether a query of `count` rays on this scene is walked in key order under the current
 * pt_query_order setting (*ordered = 1: a key kernel and a radix sort run before the walk). */
pt_status pt_query_ordered(const pt_scene *scene, size_t count, int *ordered);

/* ---- ray queries ----
 * Closest hit follows trace_world(…, brute=false) (src/renderer/transport.h:43-85) with
 * exact-distance ties resolved to the lowest (primitive_type, primitive_id); any-hit answers
 * whether a primitive is hit in (tmin, tmax), the question trace_color's shadow query asks
 * (src/renderer/transport.h:206-209). */
enum { PT_QUERY_CLOSEST = 0, PT_QUERY_ANY = 1 };
/* Device buffers, asynchronous on `stream` (a cudaStream_t; 0 = legacy default stream).
 * `tmax` may be NULL (FLT_MAX for every ray); `stats` may be NULL.  Several host threads may query
 * one scene; each launch takes one of the scene's 64 ray counters in turn, so at most 64 queries of
 * one scene may be in flight on the GPU at once. */
pt_status pt_query_rays_device(const pt_scene *scene, const pt_ray *rays, size_t count, int mode,
                               float tmin, const float *tmax, pt_hit *hits, pt_ray_stats *stats,
                               void *stream);
/* Host buffers: uploads, traces and downloads in overlapped chunks (2^20 rays each, on three
 * streams; the copies overlap the walk only from pinned host memory); returns when `hits` is
 * filled.  Calls on one scene from several host threads take turns (the staging buffers are the
 * scene's). */
pt_status pt_query_rays(const pt_scene *scene, const pt_ray *rays, size_t count, int mode,
                        float tmin, const float *tmax, pt_hit *hits, pt_ray_stats *stats);
/* Host-buffer query that allocates nothing.  Some callers cannot let a library call cudaMalloc
 * or cudaFree: applications that hand all device memory to their own pool allocator at start-up,
 * latency-critical loops (cudaFree can synchronize the whole device and stall other streams),
 * and processes running under a device-memory cap where a late allocation may fail.
 * No counterpart in the reference.  It walks with the process-wide settings of pt_query_layout,
 * pt_query_walk and pt_query_tuning (never in key order: see pt_query_order) and gives the
 * answers of pt_query_rays (the per-ray counters of a persistent walk depend on which rays share
 * a warp, so they may differ between calls).  It stages the rays,
 * tmax values, hits and counters through one static device array of the library (about 3.7 MB,
 * held by every GPU that loads the library until the process exits), so a call takes at most
 * PT_STATIC_QUERY_MAX_RAYS rays (more is PT_INVALID_ARGUMENT) and waits for its own work on
 * `stream` (a cudaStream_t; 0 = legacy default stream) before returning.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with that device current.
 * Every call shares the array: calls that overlap on the GPU (other streams, other host threads)
 * race on it. */
#define PT_STATIC_QUERY_MAX_RAYS 65536
pt_status pt_query_rays_static(const pt_scene *scene, const pt_ray *rays, size_t count, int mode,
                               float tmin, const float *tmax, pt_hit *hits, pt_ray_stats *stats, void *stream);
/* Compatibility form of cuda_query_rays(scene, rays, brute) (src/cuda/cuda_renderer.cu:248-260):
 * host rays in, full 56-byte trace_result records out, t range (0.001, FLT_MAX).
 * brute != 0 scans every leaf in node-array order (src/renderer/transport.h:48-60). */
pt_status pt_query_rays_compat(const pt_scene *scene, const pt_ray *rays, size_t count, int brute,
                               pt_trace_result *results);
/* trace_world(…, brute = true) (src/renderer/transport.h:48-60): every leaf in node-array order,
 * no pruning, same answer and tie rule as pt_query_rays_device.  Device buffers. */
pt_status pt_query_rays_brute_device(const pt_scene *scene, const pt_ray *rays, size_t count, int mode,
                                     float tmin, const float *tmax, pt_hit *hits, pt_ray_stats *stats,
                                     void *stream);

/* Tuning of the ray-query kernel (process-wide): persistent = 1 runs a fixed grid of warps that
 * take rays from a global counter and refill lanes whose ray has ended once fewer than
 * `min_active` (1..32) lanes are busy; persistent = 0 launches one thread per ray.
 * blocks_per_sm = 0 uses the occupancy limit.  Defaults: 1, 24, 0. */
pt_status pt_query_tuning(int persistent, int min_active, int blocks_per_sm);
/* Node layout of the traversal kernels (process-wide; renderers pick it up when created):
 * 1 = four-wide nodes (up to 4 primitives per leaf) where the scene's tree allows it (default),
 * 0 = the two-wide re-layout of the caller's tree.  A renderer of a tree of at most 32 four-wide
 * nodes walks the two-wide layout either way (faster on so few nodes).  Results do not depend
 * on it. */
pt_status pt_query_layout(int wide);
/* Four-wide walk form (process-wide): 1 = separate node and leaf phases per warp round, lanes
 * that already hold a leaf walking on speculatively (default); 0 = nodes and leaves in one loop. */
pt_status pt_query_walk(int speculative);
/* Ray ordering (process-wide): 1 = batches of at least 2^18 rays are walked in the order of a key
 * made of the direction's octant and a Morton code of the origin (a stable sort; lanes of a warp
 * then walk neighbouring rays), answers written back in the caller's order; 0 = rays are taken as
 * given; 2 = ordered only when the scene's walked arrays (nodes, triangle and sphere records) are
 * larger than the device's L2, where the ordering's better locality pays for the sort (default).
 * Other values are PT_INVALID_ARGUMENT.  Results do not depend on it.  pt_query_rays_static never
 * reorders. */
pt_status pt_query_order(int mode);

/* Timing of the traversal kernel alone: launches > 0 records a pair of CUDA events around each
 * of the scene's next walk-kernel launches (a ring of `launches` pairs; 0 stops recording), and
 * pt_query_profile_read returns their durations in ms, oldest first (waits for the last one). */
pt_status pt_query_profile(pt_scene *scene, int launches);
pt_status pt_query_profile_read(pt_scene *scene, float *ms, size_t capacity, size_t *count);
/* Read bandwidth of this GPU in GB/s for a buffer of `bytes` read `reps` times with 16-byte loads
 * (under the L2 size: L2 bandwidth; several GB: HBM); allocates and frees the buffer. */
pt_status pt_probe_read_bandwidth(size_t bytes, int reps, float *gbs);

/* ---- device ray generators (bit-identical to the host ones in pt_workloads.h) ----
 * Camera rays of pt_rays_camera; bounce rays from closest hits: origin at the hit, a
 * cosine-distributed direction about the geometric normal turned toward the ray, one PCG stream
 * per ray seeded (seed, first + k); a primary miss becomes a random surface ray. */
pt_status pt_rays_camera_device(const pt_camera *camera, int width, int height, uint64_t seed, uint64_t first,
                                size_t count, pt_ray *rays, void *stream);
pt_status pt_rays_bounce_device(const pt_scene *scene, const pt_ray *primary, const pt_hit *hits, size_t count,
                                uint64_t seed, uint64_t first, pt_ray *rays, void *stream);
/* Surface rays of pt_rays_surface (pt_workloads.h) on the device: stream (seed, first + k) per ray;
 * shadow_tmax non-NULL: shadow rays between two surface points with shadow_tmax[k] = distance - 0.001. */
pt_status pt_rays_surface_device(const pt_scene *scene, uint64_t seed, uint64_t first, size_t count, pt_ray *rays,
                                 float *shadow_tmax, void *stream);

/* ---- progressive renderer ----
 * Replaces class cuda_renderer (src/cuda/cuda_renderer.h:10-29).  `flags` is a bit set of
 * PT_RENDER_*; `max_depth` is the last bounce index of trace_color's loop (the reference
 * hard-codes 50, src/renderer/transport.h:174,193). */
enum { PT_RENDER_MIS = 1, PT_RENDER_BRUTE = 2 };
pt_status pt_renderer_create(const pt_scene *scene, const pt_camera *camera, int width, int height,
                             uint64_t seed, uint32_t flags, int debug_mode, int max_depth,
                             pt_renderer **out);
pt_status pt_renderer_destroy(pt_renderer *renderer);
/* reset(camera): zero the sums, reseed every pixel's PCG stream (src/cuda/cuda_renderer.cu:186-194). */
pt_status pt_reset(pt_renderer *renderer, const pt_camera *camera);
/* add_samples(count) (src/cuda/cuda_renderer.cu:196-213); blocks until the samples are done. */
pt_status pt_add_samples(pt_renderer *renderer, int count);
/* set_block_shape(w, h): accepted shapes 8x8, 16x8, 16x16, 32x8 (src/cuda/cuda_renderer.cu:215-228).
 * Sets the thread-block size of the wavefront kernels to w*h threads. */
pt_status pt_set_block_shape(pt_renderer *renderer, int width, int height);
/* Live-path count below which add_samples stops the wavefront and runs the remaining paths to
 * completion in one fused kernel (two threads per path on four-wide trees: one walks the path's
 * next ray while the other walks its last shadow ray; default max(65536, pixels/4); 0 keeps the
 * wavefront to the end).  Results do not depend on it. */
pt_status pt_renderer_tuning(pt_renderer *renderer, int32_t tail_paths);
/* Linear FP32 radiance sums (3 floats per pixel, row 0 at the bottom, not divided by spp). */
pt_status pt_get_sums(const pt_renderer *renderer, float *rgb_sums, size_t floats);
/* image(): sums / spp (src/cuda/cuda_renderer.cu:230-234). */
pt_status pt_get_image(const pt_renderer *renderer, float *rgb, size_t floats);
/* Per-pixel PCG-XSH-RR states as (state, increment) pairs (src/renderer/random.h:8-23). */
pt_status pt_get_rng(const pt_renderer *renderer, uint64_t *state_increment_pairs, size_t words);
/* write_rgba(device_ptr, bytes): gamma-2 RGBA8 packing (src/cuda/cuda_renderer.cu:99-109, 235-240). */
pt_status pt_write_rgba(const pt_renderer *renderer, unsigned char *device_pixels, size_t bytes);
/* rgba_image(): same bytes, into host memory. */
pt_status pt_rgba_image(const pt_renderer *renderer, unsigned char *host_pixels, size_t bytes);
/* sample_count(), kernel_milliseconds(), rays_traced(). */
pt_status pt_stats(const pt_renderer *renderer, int *samples, float *kernel_ms, uint64_t *rays);

/* ---- batched rendering ----
 * Many render jobs — each its own scene, camera, resolution, sample count, bounce limit and seed —
 * rendered together: every job's scene is merged into one device scene and a pool of path slots
 * walks all jobs' pixels inside one CUDA graph launch (a device-side loop of wavefront
 * iterations, then a fused kernel for the tail).  Each job's sums equal those of a pt_renderer
 * rendering that job alone (MIS flag as given, debug views not supported).  No counterpart in the
 * reference, which renders one image per cuda_renderer. */
typedef struct pt_job {
    int32_t scene;              /* index into the scene list of pt_batch_create */
    int32_t width, height, samples, max_depth;
    uint64_t seed;
    pt_camera camera;
} pt_job;
typedef struct pt_batch pt_batch;
pt_status pt_batch_create(const pt_scene_desc *scenes, int32_t scene_count, const pt_job *jobs, int32_t job_count,
                          uint32_t flags, pt_batch **out);
pt_status pt_batch_destroy(pt_batch *batch);
/* Renders every job's samples from a fresh state (sums zeroed, streams seeded); blocks. */
pt_status pt_batch_run(pt_batch *batch);
pt_status pt_batch_get_sums(const pt_batch *batch, int32_t job, float *rgb_sums, size_t floats);
/* Device time of the last run, rays traced, and each job's completion time from the run's start. */
pt_status pt_batch_stats(const pt_batch *batch, float *kernel_ms, uint64_t *rays, double *job_completion_ms, size_t jobs);
/* path_capacity: path slots (0 = min(pixels, 2^22)); block: 64, 128 or 256 threads; min_active:
 * traversal refill threshold; tail_paths: live paths below which the fused kernel finishes;
 * use_graph: 1 = one graph launch with a device-side loop, 0 = host-driven loop. */
pt_status pt_batch_tuning(pt_batch *batch, int32_t path_capacity, int32_t block, int32_t min_active, int32_t tail_paths,
                          int32_t use_graph);
/* Node fetch width of the batch's walks: 1 = four-wide nodes (default), 0 = the two-wide layout.
 * Results do not depend on it. */
pt_status pt_batch_node_width(pt_batch *batch, int32_t wide);
/* Sweeps capacity x block x min_active x graph on probe runs (each job at min(probe_samples, its
 * samples)), then the other node fetch width at the fastest of those, applies the fastest and caches
 * it per (log2 triangles, log2 pixels) bucket in `cache_path` (NULL: no cache).  best (5 entries) =
 * {capacity, block, min_active, use_graph, node_width}.  A probe run that
 * fails (timeout, stack overflow) skips its setting; the jobs' sample counts are restored whatever
 * happens; a CUDA error ends the sweep with PT_CUDA_ERROR. */
pt_status pt_batch_autotune(pt_batch *batch, int32_t probe_samples, const char *cache_path, int32_t *best);
/* Fault injection for tests, on the host: the n-th probe run of the next pt_batch_autotune fails as a
 * timed-out run would (the sweep skips that setting; the jobs keep their sample counts); n <= 0: none. */
pt_status pt_batch_fail_probe(pt_batch *batch, int32_t n);

/* ---- learned radiance cache ----
 * A small MLP (64 encoded inputs -> 5 hidden layers of 64, ReLU -> 3 outputs, exp) trained
 * online on radiance samples and queried for the outgoing radiance at a path vertex.  Forward
 * and backward run on the tensor cores (tcgen05, BF16 operands, FP32 accumulation in TMEM);
 * Adam updates FP32 master weights.  Inputs: position (frequency-encoded over the scene box, 3 x
 * 12), direction (spherical harmonics up to degree 3, 16), normal, albedo, roughness (7).
 * Loss: relative L2, mean over samples and channels of (y - t)^2 / (y^2 + 0.01) with y treated
 * as a constant in the denominator.  No counterpart in the reference. */
typedef struct pt_cache_query { pt_vec3 position, direction, normal, albedo; float roughness; } pt_cache_query;
typedef struct pt_cache pt_cache;
#define PT_CACHE_WEIGHTS 20672   /* FP32 masters: W0..W4 (64 x 64, [in][out]) then W5 (64 x 3) */
pt_status pt_cache_create(const float scene_lo[3], const float scene_hi[3], uint64_t seed, pt_cache **out);
pt_status pt_cache_destroy(pt_cache *cache);
/* rgb[3 * i] = prediction for queries[i]; device buffers, asynchronous on `stream`. */
pt_status pt_cache_query_device(pt_cache *cache, const pt_cache_query *queries, size_t count, float *rgb, void *stream);
/* One Adam step on (queries, targets) (device buffers).  loss == NULL: asynchronous on `stream`;
 * otherwise the call waits and *loss = the batch's mean loss. */
pt_status pt_cache_train_device(pt_cache *cache, const pt_cache_query *queries, const float *targets, size_t count,
                                float *loss, void *stream);
/* The gradient of the mean loss w.r.t. the FP32 masters (host buffer of PT_CACHE_WEIGHTS), no update. */
pt_status pt_cache_gradients(pt_cache *cache, const pt_cache_query *queries, const float *targets, size_t count,
                             float *grad, float *loss);
/* Waits for `stream`; returns PT_TIMEOUT (and clears it) when a tensor-core wait of an earlier
 * asynchronous call of this cache ran out (its outputs are then not valid and no Adam step was
 * applied).  Every wait of the cache's kernels is bounded; after one runs out the kernel waits once
 * more, with the full bound, for the tensor-core work it had issued, frees its TMEM and returns. */
pt_status pt_cache_sync(pt_cache *cache, void *stream);
/* try_wait attempts per bounded wait of this cache's kernels (< 0: the default, 2^22).  0 makes every
 * wait run out at once: fault injection for tests of the PT_TIMEOUT path. */
pt_status pt_cache_wait_limit(pt_cache *cache, long long attempts);
/* Reads (get != NULL) and/or replaces (set != NULL) the FP32 master weights. */
pt_status pt_cache_weights(pt_cache *cache, float *get, const float *set, size_t floats);
/* Adam hyper-parameters (defaults 1e-2, 0.9, 0.99, 1e-8). */
pt_status pt_cache_hyper(pt_cache *cache, float lr, float beta1, float beta2, float eps);
/* decay > 0: every Adam step also updates an exponential moving average of the weights
 * (bias-corrected) and queries use the average; 0 (the default): queries use the weights.
 * Restarts the average from the current weights. */
pt_status pt_cache_average(pt_cache *cache, float decay);

/* ---- radiance-cache renderer ----
 * Renders frames of one sample per pixel with MIS (the shading of the plain renderer) and ends
 * each path at its first diffuse vertex whose path spread exceeds `spread_threshold` times the
 * primary footprint (the area-spread heuristic of neural radiance caching): the pixel gets the
 * path's radiance so far plus throughput x albedo x the network's prediction there.  About
 * `training_paths` pixels per frame (chosen by a hash of seed, frame and pixel) trace on for
 * `suffix_bounces` more bounces and end at the cache; the radiance they collect after each
 * diffuse vertex, divided by its albedo, is a training target, and `train_steps` Adam steps per
 * frame fit the network to them.  A frame is one CUDA graph launch.  No counterpart in the
 * reference; use_cache = 0 gives the plain path tracer through the same kernels. */
typedef struct pt_cached_params {
    int32_t training_paths;     /* per frame (default 65536) */
    int32_t train_steps;        /* Adam steps per frame (1); the training samples are split between them */
    int32_t suffix_bounces;     /* bounces traced beyond the query by training paths (4, at most 8) */
    int32_t use_cache;          /* 1: end paths at the cache; 0: plain path tracing */
    int32_t train;              /* 1: online training; 0: the network stays as it is */
    int32_t use_graph;          /* 1: one graph launch per frame; 0: the same kernels launched one by one */
    float spread_threshold;     /* c of the termination rule (0.3) */
    float learning_rate;        /* Adam learning rate (1e-2; beta 0.9 / 0.99) */
    uint64_t network_seed;      /* weight initialisation */
    int32_t tail_paths;         /* live paths below which one fused kernel ends the frame's tail
                                 * (0: max(16384, pixels / 16)) */
    int32_t query_specular;     /* 1 (default): paths may also end at metal and glass vertices;
                                 * 0: at diffuse vertices only */
    float weight_average;       /* decay of the weight average queries use (0.99; 0: the live weights) */
    int32_t samples_per_frame;  /* samples per pixel in one frame (4; 1..64); the network trains once per frame */
} pt_cached_params;
typedef struct pt_cached_renderer pt_cached_renderer;
/* params == NULL: the defaults above. */
pt_status pt_cached_defaults(pt_cached_params *params);
pt_status pt_cached_create(const pt_scene *scene, const pt_camera *camera, int width, int height, uint64_t seed, int max_depth,
                           const pt_cached_params *params, pt_cached_renderer **out);
pt_status pt_cached_destroy(pt_cached_renderer *renderer);
/* `frames` frames; accumulate = 0: training-only frames (only the training paths are traced, one
 * sample each, and the image is left alone), 1: every pixel is rendered with samples_per_frame
 * samples and added to the image sums. */
pt_status pt_cached_frames(pt_cached_renderer *renderer, int frames, int accumulate);
/* on = 0: later frames leave the network as it is (and trace no training paths); 1: online
 * training again (when the renderer was created with training). */
pt_status pt_cached_training(pt_cached_renderer *renderer, int on);
/* Clears the image sums and frame count (the network and the pixels' RNG streams go on). */
pt_status pt_cached_clear(pt_cached_renderer *renderer);
pt_status pt_cached_get_sums(const pt_cached_renderer *renderer, float *rgb, size_t floats);
/* frames: accumulated samples per pixel; kernel_ms: device time of all frames; rays: closest-hit + shadow
 * queries; queries: cache queries; samples: training samples; loss: mean loss of the last step. */
pt_status pt_cached_stats(pt_cached_renderer *renderer, int *frames, float *kernel_ms, uint64_t *rays, uint64_t *queries,
                          uint64_t *samples, float *loss);
/* The renderer's network (owned by the renderer; valid until pt_cached_destroy). */
pt_status pt_cached_cache(pt_cached_renderer *renderer, pt_cache **cache);

#ifdef __cplusplus
}
#endif

#endif
