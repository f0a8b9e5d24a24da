// pt_batch.cu — many render jobs (uneven resolutions, scenes, spp, bounce limits) in one launch.
//
// The reference renders one image per cuda_renderer and one add_samples launch at a time
// (src/cuda/cuda_renderer.cu:196-213).  Here every job's scene is merged into one device scene
// (one four-wide node array with a root per job, one slot space, offset material/texture/light
// indices), and a fixed pool of path slots walks all jobs' pixels: a slot renders one pixel's
// samples in order (so each pixel's PCG stream is consumed exactly as a lone renderer would) and
// then takes the next pixel from a global cursor.  One CUDA graph runs the whole batch: a
// conditional WHILE node whose body is two wavefront iterations (extend, shade, shadow) and a
// one-thread control kernel that decides from the live-path count whether to go on, then the
// fused finish kernel for the short tail.  Per-job completion times come from %globaltimer.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include "pt_api_common.h"
#include "pt_device.h"
#include "pt_wavefront.h"

using namespace ptb;

namespace ptb {

struct BatchJob {
    pt_camera camera;
    int32_t width, height, samples, max_depth;
    uint64_t seed;
    int64_t pixel_offset;
    int32_t pixel_count, root;        // root: the job's tree in the four-wide node array (-1: empty)
    int32_t light_offset, light_count;
    float light_area;
    int32_t root2;                    // the job's tree in the two-wide node array (-1: empty)
};

struct BatchBuffers {
    const BatchJob *jobs;
    int32_t job_count;
    int64_t total_pixels;
    int mis;
    float *sums;
    Pcg *rng;
    PathState *paths;
    PathHit *hits;
    ShadowRay *shadows;
    int64_t *slot_pixel;
    int32_t *slot_job;
    int32_t *queue[2];
    int32_t *shadow_queue;
    int32_t *counters;                // [0],[1] path queues, [2],[3] shadow queues of even and odd iterations
    unsigned long long *fetch;        // [0] extend items, [1],[2] shadow items of even and odd iterations, [3] tail slots
    unsigned long long *cursor;       // next pixel to start
    unsigned long long *rays;
    int32_t *job_remaining;
    unsigned long long *job_done_ns;
    unsigned long long *start_ns;
    int32_t *error;
    unsigned long long *iterations;
};

__device__ inline unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ inline int32_t job_of(const BatchBuffers &b, int64_t pixel) {
    int32_t lo = 0, hi = b.job_count - 1;
    while (lo < hi) {
        int32_t mid = (lo + hi + 1) / 2;
        if (b.jobs[mid].pixel_offset <= pixel) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ inline ShadeCtx job_ctx(const BatchJob &j, int mis) {
    ShadeCtx c;
    c.camera = &j.camera; c.width = j.width; c.height = j.height; c.max_depth = j.max_depth;
    c.debug = PT_DEBUG_SHADED; c.mis = mis;
    return c;
}

// The merged scene seen by one job: its own emitter table.
__device__ inline DeviceScene job_scene(const DeviceScene &merged, const BatchJob &j) {
    DeviceScene s = merged;
    s.lights = merged.lights + j.light_offset;
    s.light_count = j.light_count;
    s.light_area = j.light_area;
    return s;
}

// initialize_pixels per job: zero sums, seed each pixel's stream with (job seed, pixel index).
__global__ void batch_init(BatchBuffers b) {
    int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= b.total_pixels) return;
    const BatchJob &j = b.jobs[job_of(b, g)];
    b.sums[3 * g] = 0; b.sums[3 * g + 1] = 0; b.sums[3 * g + 2] = 0;
    Pcg r; r.seed(j.seed, uint64_t(g - j.pixel_offset));
    b.rng[g] = r;
}

// A slot starts pixel g: its first camera ray.
__device__ inline void start_pixel(const BatchBuffers &b, int32_t slot, int64_t g, PathState &s) {
    int32_t jid = job_of(b, g);
    const BatchJob &j = b.jobs[jid];
    Pcg rng = b.rng[g];
    camera_path(j.camera, j.width, j.height, int32_t(g - j.pixel_offset), rng, s);
    s.samples_left = j.samples;
    b.rng[g] = rng;
    b.slot_pixel[slot] = g;
    b.slot_job[slot] = jid;
}

__global__ void batch_start(BatchBuffers b, int32_t slots) {
    int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) {
        b.counters[0] = slots; b.counters[1] = 0; b.counters[2] = 0; b.counters[3] = 0;
        b.fetch[0] = 0; b.fetch[1] = 0; b.fetch[2] = 0; b.fetch[3] = 0;
        *b.cursor = (unsigned long long)slots;
        *b.start_ns = globaltimer();
        *b.iterations = 0;
    }
    if (k >= slots) return;
    PathState s;
    start_pixel(b, k, k, s);
    b.paths[k] = s;
    b.queue[0][k] = k;
}

// kWide: four-wide nodes (phased walk) or the two-wide layout.
template <bool kWide>
__global__ void __launch_bounds__(256, 4) batch_extend(DeviceScene scene, BatchBuffers b, int parity, int min_active) {
    const int32_t n = b.counters[parity];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(b.rays, (unsigned long long)n);
        b.counters[parity ^ 1] = 0;
        b.counters[2 + parity] = 0;      // this iteration's shadow slot (the other may be in use)
        b.fetch[1 + parity] = 0;
    }
    const int32_t *queue = b.queue[parity];
    auto get = [&](size_t k, pt_ray &r, float &lo, float &hi, int32_t &root) {
        int32_t slot = queue[k];
        r = path_ray(b.paths[slot]);
        lo = 0.001f; hi = FLT_MAX;
        const BatchJob &j = b.jobs[b.slot_job[slot]];
        root = kWide ? j.root : j.root2;
    };
    auto done = [&](size_t k, const WalkResult &w) {
        if (w.error) *b.error = 1;
        PathHit out;
        out.t = w.t; out.u = w.u; out.v = w.v; out.slot = w.error ? -2 : w.slot;
        b.hits[queue[k]] = out;
    };
    if constexpr (kWide) persistent_walk4_spec<false, true>(scene, size_t(n), &b.fetch[0], min_active, kTieLastLeaf, get, done);
    else persistent_walk<false, true>(scene, size_t(n), &b.fetch[0], min_active, kTieLastLeaf, get, done);
}

__global__ void batch_shade(DeviceScene scene, BatchBuffers b, int parity) {
    const int32_t n = b.counters[parity];
    const int32_t *in = b.queue[parity];
    int32_t *out = b.queue[parity ^ 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) b.fetch[0] = 0;
    for (int32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        int32_t k = base + threadIdx.x;
        bool valid = k < n, live = false, shadow = false;
        int32_t slot = valid ? in[k] : 0;
        bool finished_pixel = false;
        PathState s;
        if (valid) {
            s = b.paths[slot];
            PathHit h = b.hits[slot];
            int64_t g = b.slot_pixel[slot];
            int32_t jid = b.slot_job[slot];
            const BatchJob &j = b.jobs[jid];
            DeviceScene js = job_scene(scene, j);
            Pcg rng = b.rng[g];
            ShadowRay sr;
            live = shade_path(js, job_ctx(j, b.mis), b.sums + 3 * g, int32_t(g - j.pixel_offset), slot, s, h, make_uint2(0, 0),
                              rng, sr, shadow);
            b.rng[g] = rng;
            if (shadow) b.shadows[slot] = sr;
            if (!live) {
                finished_pixel = true;
                if (atomicSub(&b.job_remaining[jid], 1) == 1) b.job_done_ns[jid] = globaltimer();
            }
        }
        // slots whose pixel is done take the next pixel (one atomicAdd per warp)
        unsigned m = __ballot_sync(0xffffffffu, finished_pixel);
        if (m) {
            int leader = __ffs(m) - 1;
            unsigned long long first = 0;
            if ((int)lane_id() == leader) first = atomicAdd(b.cursor, (unsigned long long)__popc(m));
            first = __shfl_sync(0xffffffffu, first, leader);
            if (finished_pixel) {
                unsigned long long g = first + __popc(m & ((1u << lane_id()) - 1u));
                if (g < (unsigned long long)b.total_pixels) { start_pixel(b, slot, int64_t(g), s); live = true; }
            }
        }
        if (valid) b.paths[slot] = s;
        push(live, slot, out, &b.counters[parity ^ 1]);
        push(shadow, slot, b.shadow_queue, &b.counters[2 + parity]);
    }
}

template <bool kWide>
__global__ void __launch_bounds__(256, 4) batch_shadow(DeviceScene scene, BatchBuffers b, int parity, int min_active) {
    const int32_t n = b.counters[2 + parity];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(b.rays, (unsigned long long)n);
    auto get = [&](size_t k, pt_ray &r, float &lo, float &hi, int32_t &root) {
        int32_t slot = b.shadow_queue[k];
        const ShadowRay &sr = b.shadows[slot];
        r.origin = pt_vec3{sr.ox, sr.oy, sr.oz};
        r.direction = pt_vec3{sr.dx, sr.dy, sr.dz};
        r.time = sr.time;
        lo = 0.001f; hi = sr.tmax;
        const BatchJob &j = b.jobs[b.slot_job[slot]];
        root = kWide ? j.root : j.root2;
    };
    auto done = [&](size_t k, const WalkResult &w) {
        if (w.error) { *b.error = 1; return; }
        if (w.slot < 0) {
            int32_t slot = b.shadow_queue[k];
            const ShadowRay &sr = b.shadows[slot];
            PathState &s = b.paths[slot];
            s.rr = s.rr + sr.cr; s.rg = s.rg + sr.cg; s.rb = s.rb + sr.cb;
        }
    };
    if constexpr (kWide) persistent_walk4_spec<true, true>(scene, size_t(n), &b.fetch[1 + parity], min_active, kTieLastLeaf, get, done);
    else persistent_walk<true, true>(scene, size_t(n), &b.fetch[1 + parity], min_active, kTieLastLeaf, get, done);
}

// One thread: continue the WHILE loop while paths are live, unless only a short tail is left
// (then the finish kernel takes it) or the iteration bound is reached (an error).
__global__ void batch_control(BatchBuffers b, cudaGraphConditionalHandle handle, int32_t tail_paths, unsigned long long max_iterations) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int32_t live = b.counters[0];
    unsigned long long it = ++*b.iterations;
    bool pixels_left = *b.cursor < (unsigned long long)b.total_pixels;
    bool go = live > 0 && (live >= tail_paths || pixels_left);
    if (go && it >= max_iterations) { *b.error = 2; go = false; }
    cudaGraphSetConditional(handle, go ? 1u : 0u);
}

// The tail, two lanes per slot: in each round the even lane of a pair walks its path's next ray
// while the odd lane walks the shadow ray of the path's previous bounce (one runtime-mode walk,
// traverse4_rt or traverse_rt), so a bounce costs one walk's latency instead of two.  The shadow contribution of
// bounce k is added before bounce k+1 is shaded, the order of the iterations above, so the sums
// are bit-identical.  A pair whose pixel is done takes the next pixel while any remain, then the next
// queued slot (fetch[3]).
template <bool kWide>
__global__ void __launch_bounds__(256, 2) batch_finish_pair(DeviceScene scene, BatchBuffers b) {
    const int32_t n = b.counters[0];
    const unsigned full = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31;
    const bool odd = lane & 1;
    const unsigned even_lane = lane & ~1u, odd_lane = lane | 1u;
    unsigned long long rays = 0;
    int32_t slot = -1;             // even lane: the slot in hand, -1 when none
    PathState s{};
    int64_t g = 0;                 // even lane: the slot's pixel
    int32_t jid = 0;
    Pcg rng{};
    bool live = false;             // even lane: the path has a ray to walk
    bool pending = false;          // even lane: a shadow ray from the last shading waits
    bool drained = false;          // even lane: neither pixels nor queued slots are left
    ShadowRay sr{};
    bool walk_shadow = false;      // odd lane: walks the pair's pending shadow ray this round
    pt_ray q{};
    float qmax = 0;
    int32_t qroot = 0;
    for (;;) {
        if (!odd && !live && !pending && !drained) {
            if (slot >= 0) {       // the pixel in hand is done
                b.rng[g] = rng;
                if (atomicSub(&b.job_remaining[jid], 1) == 1) b.job_done_ns[jid] = globaltimer();
                unsigned long long next = atomicAdd(b.cursor, 1ull);
                if (next < (unsigned long long)b.total_pixels) {
                    start_pixel(b, slot, int64_t(next), s);
                    g = int64_t(next); jid = b.slot_job[slot]; rng = b.rng[g];
                    live = true;
                } else {
                    b.paths[slot] = s;
                    slot = -1;
                }
            }
            if (slot < 0) {
                unsigned long long k = atomicAdd(&b.fetch[3], 1ull);
                if (k < (unsigned long long)n) {
                    slot = b.queue[0][k];
                    s = b.paths[slot]; g = b.slot_pixel[slot]; jid = b.slot_job[slot]; rng = b.rng[g];
                    live = true;
                } else {
                    drained = true;
                }
            }
        }
        const bool work = odd ? walk_shadow : live;   // both lanes' rounds stay in step (warp-uniform loop)
        if (!__any_sync(full, work)) break;
        const int32_t root = odd ? qroot : (live ? (kWide ? b.jobs[jid].root : b.jobs[jid].root2) : 0);
        HitInfo hi;
        uint32_t boxes = 0, prims = 0;
        int error = 0;
        bool hit = false;
        if (work) {
            rays++;
            if constexpr (kWide)
                hit = traverse4_rt(scene, odd ? q : path_ray(s), 0.001f, odd ? qmax : FLT_MAX, kTieLastLeaf, odd, hi, boxes, prims,
                                   error, root);
            else
                hit = traverse_rt(scene, odd ? q : path_ray(s), 0.001f, odd ? qmax : FLT_MAX, kTieLastLeaf, odd, hi, boxes, prims,
                                  error, root);
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
                const BatchJob &j = b.jobs[jid];
                DeviceScene js = job_scene(scene, j);
                PathHit h;
                h.t = hi.t; h.u = hi.u; h.v = hi.v; h.slot = (hit && !error) ? hi.slot : (error ? -2 : -1);
                bool shadow = false;
                live = shade_path(js, job_ctx(j, b.mis), b.sums + 3 * g, int32_t(g - j.pixel_offset), slot, s, h, make_uint2(0, 0),
                                  rng, sr, shadow);
                pending = shadow;
            }
        }
        // the even lane hands its new shadow ray (and its job's tree root) to the odd lane
        walk_shadow = __shfl_sync(full, pending, even_lane);
        q.origin.x = __shfl_sync(full, sr.ox, even_lane);
        q.origin.y = __shfl_sync(full, sr.oy, even_lane);
        q.origin.z = __shfl_sync(full, sr.oz, even_lane);
        q.direction.x = __shfl_sync(full, sr.dx, even_lane);
        q.direction.y = __shfl_sync(full, sr.dy, even_lane);
        q.direction.z = __shfl_sync(full, sr.dz, even_lane);
        q.time = __shfl_sync(full, sr.time, even_lane);
        qmax = __shfl_sync(full, sr.tmax, even_lane);
        qroot = __shfl_sync(full, root, even_lane);
    }
    for (int o = 16; o; o >>= 1) rays += __shfl_down_sync(full, rays, o);
    if (lane == 0 && rays) atomicAdd(b.rays, rays);
}

} // namespace ptb

namespace ptb {
// Four pinned host words for the host-driven loop's read-backs, freed on every path out.
struct PinnedWords {
    int32_t *words = nullptr;
    PinnedWords() { PT_CUDA(cudaMallocHost(&words, 4 * sizeof(int32_t))); }
    ~PinnedWords() { if (words) cudaFreeHost(words); }
    PinnedWords(const PinnedWords &) = delete;
    PinnedWords &operator=(const PinnedWords &) = delete;
};
} // namespace ptb

struct pt_batch {
    DeviceScene view{};
    DeviceBuffer nodes4, nodes2, tris, spheres, triangles, sphere_src, materials, textures, pixels, lights, jobs;
    DeviceBuffer sums, rng, paths, hits, shadows, slot_pixel, slot_job, queue0, queue1, shadow_queue, counters, fetch, scalars,
        job_remaining, job_done_ns, error;
    std::vector<BatchJob> host_jobs;
    int64_t total_pixels = 0;
    uint64_t total_triangles = 0;
    int mis = 1;
    // tuning (pt_batch_tuning / pt_batch_autotune)
    int32_t capacity = 0, block = 256, min_active = 16, tail_paths = 16384, use_graph = 1;
    int32_t wide = 1;                     // node fetch width: 1 four-wide nodes, 0 the two-wide layout
    int32_t probe_fault_countdown = 0;   // > 0: that autotune probe run fails on the host (tests)
    int32_t slots = 0;
    BatchBuffers buf{};
    cudaStream_t stream = nullptr;
    cudaStream_t shadow_stream = nullptr;   // a shadow kernel runs beside the next extend
    Event shaded[2], shadowed[2];
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    Event start, stop;
    float milliseconds = 0;
    uint64_t rays = 0;
    std::vector<double> job_ms;
    ~pt_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (shadow_stream) cudaStreamDestroy(shadow_stream);
        if (stream) cudaStreamDestroy(stream);
    }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr; graph = nullptr;
    }
    size_t stack_smem() const {
        return wide ? size_t(kSharedStack4) * sizeof(int2) * size_t(block) : size_t(kSharedStack) * sizeof(int32_t) * size_t(block);
    }
    const void *extend_fn() const { return wide ? (const void *)batch_extend<true> : (const void *)batch_extend<false>; }
    const void *shadow_fn() const { return wide ? (const void *)batch_shadow<true> : (const void *)batch_shadow<false>; }
    const void *finish_fn() const { return wide ? (const void *)batch_finish_pair<true> : (const void *)batch_finish_pair<false>; }
    void launch_finish(cudaStream_t st) {
        if (wide) batch_finish_pair<true><<<grid(finish_fn(), 0), block, 0, st>>>(view, buf);
        else batch_finish_pair<false><<<grid(finish_fn(), 0), block, 0, st>>>(view, buf);
    }
    int grid(const void *fn, size_t smem) const {
        int per_sm = 0;
        PT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem));
        return device_sm_count() * (per_sm > 0 ? per_sm : 1);
    }
    void allocate_slots() {
        int32_t want = capacity > 0 ? capacity : int32_t(std::min<int64_t>(total_pixels, 1 << 22));
        slots = int32_t(std::min<int64_t>(want, total_pixels));
        size_t n = size_t(std::max(slots, 1));
        paths.resize(n * sizeof(PathState)); hits.resize(n * sizeof(PathHit)); shadows.resize(n * sizeof(ShadowRay));
        slot_pixel.resize(n * sizeof(int64_t)); slot_job.resize(n * sizeof(int32_t));
        queue0.resize(n * sizeof(int32_t)); queue1.resize(n * sizeof(int32_t)); shadow_queue.resize(n * sizeof(int32_t));
        buf.paths = paths.get<PathState>(); buf.hits = hits.get<PathHit>(); buf.shadows = shadows.get<ShadowRay>();
        buf.slot_pixel = slot_pixel.get<int64_t>(); buf.slot_job = slot_job.get<int32_t>();
        buf.queue[0] = queue0.get<int32_t>(); buf.queue[1] = queue1.get<int32_t>(); buf.shadow_queue = shadow_queue.get<int32_t>();
        drop_graph();
    }
    unsigned long long max_iterations() const {
        // every pixel needs at most samples * (depth + 1) extends; slots run pixels back to back
        unsigned long long worst = 0;
        for (const auto &j : host_jobs) worst = std::max<unsigned long long>(worst, (unsigned long long)j.samples * (j.max_depth + 1));
        unsigned long long waves = (unsigned long long)((total_pixels + slots - 1) / std::max(slots, 1)) + 1;
        return worst * waves + 16;
    }
    // Two wavefront iterations.  The first one's shadow kernel runs on the shadow stream beside
    // the second one's extend; shade waits for the shadow kernel before it (it rewrites the
    // shadow records and reads the radiance the shadow kernel adds); the pair ends joined.
    void pair(cudaStream_t st) {
        const size_t smem = stack_smem();
        for (int parity = 0; parity < 2; parity++) {
            if (wide) batch_extend<true><<<grid(extend_fn(), smem), block, smem, st>>>(view, buf, parity, min_active);
            else batch_extend<false><<<grid(extend_fn(), smem), block, smem, st>>>(view, buf, parity, min_active);
            if (parity == 1) PT_CUDA(cudaStreamWaitEvent(st, shadowed[0].get(), 0));
            batch_shade<<<grid((const void *)batch_shade, 0), block, 0, st>>>(view, buf, parity);
            PT_CUDA(cudaEventRecord(shaded[parity].get(), st));
            PT_CUDA(cudaStreamWaitEvent(shadow_stream, shaded[parity].get(), 0));
            if (wide) batch_shadow<true><<<grid(shadow_fn(), smem), block, smem, shadow_stream>>>(view, buf, parity, min_active);
            else batch_shadow<false><<<grid(shadow_fn(), smem), block, smem, shadow_stream>>>(view, buf, parity, min_active);
            PT_CUDA(cudaEventRecord(shadowed[parity].get(), shadow_stream));
        }
        PT_CUDA(cudaStreamWaitEvent(st, shadowed[1].get(), 0));
        PT_CUDA(cudaGetLastError());
    }
    void build_graph() {
        drop_graph();
        PT_CUDA(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle handle;
        PT_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t loop;
        PT_CUDA(cudaGraphAddNode(&loop, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        PT_CUDA(cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        pair(stream);
        batch_control<<<1, 32, 0, stream>>>(buf, handle, tail_paths, max_iterations());
        PT_CUDA(cudaStreamEndCapture(stream, &body));
        PT_CUDA(cudaStreamBeginCaptureToGraph(stream, graph, &loop, nullptr, 1, cudaStreamCaptureModeRelaxed));
        launch_finish(stream);
        PT_CUDA(cudaStreamEndCapture(stream, &graph));
        PT_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    }
    void run() {
        cudaStream_t st = stream;
        int32_t njobs = int32_t(host_jobs.size());
        std::vector<int32_t> remaining(static_cast<size_t>(njobs));
        for (int32_t k = 0; k < njobs; k++) remaining[size_t(k)] = host_jobs[size_t(k)].pixel_count;
        PT_CUDA(cudaMemcpyAsync(buf.job_remaining, remaining.data(), remaining.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        PT_CUDA(cudaMemsetAsync(buf.job_done_ns, 0, size_t(njobs) * sizeof(unsigned long long), st));
        PT_CUDA(cudaMemsetAsync(buf.rays, 0, sizeof(unsigned long long), st));
        PT_CUDA(cudaMemsetAsync(buf.error, 0, sizeof(int32_t), st));
        batch_init<<<unsigned((total_pixels + 255) / 256), 256, 0, st>>>(buf);
        PT_CUDA(cudaEventRecord(start.get(), st));
        batch_start<<<(slots + 255) / 256, 256, 0, st>>>(buf, slots);
        PT_CUDA(cudaGetLastError());
        if (use_graph) {
            if (!exec) build_graph();
            PT_CUDA(cudaGraphLaunch(exec, st));
        } else {
            // host-driven form of the same loop: iterations in pairs, live count read back each pair
            unsigned long long bound = max_iterations();
            PinnedWords live_host;
            unsigned long long cursor = 0;
            for (unsigned long long it = 0;; it++) {
                pair(st);
                PT_CUDA(cudaMemcpyAsync(live_host.words, buf.counters, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
                PT_CUDA(cudaMemcpyAsync(&cursor, buf.cursor, sizeof cursor, cudaMemcpyDeviceToHost, st));
                PT_CUDA(cudaStreamSynchronize(st));
                int32_t live = live_host.words[0];
                if (live == 0 || (live < tail_paths && cursor >= (unsigned long long)total_pixels)) break;
                if (it + 1 >= bound) throw Error(PT_TIMEOUT, "batch did not drain within its iteration bound");
            }
            launch_finish(st);
        }
        PT_CUDA(cudaGetLastError());
        PT_CUDA(cudaEventRecord(stop.get(), st));
        PT_CUDA(cudaEventSynchronize(stop.get()));
        int32_t error = 0;
        PT_CUDA(cudaMemcpy(&error, buf.error, sizeof error, cudaMemcpyDeviceToHost));
        if (error == 1) throw Error(PT_STACK_OVERFLOW, "CUDA traversal stack overflow");
        if (error == 2) throw Error(PT_TIMEOUT, "batch did not drain within its iteration bound");
        PT_CUDA(cudaEventElapsedTime(&milliseconds, start.get(), stop.get()));
        unsigned long long total = 0, t0 = 0;
        PT_CUDA(cudaMemcpy(&total, buf.rays, sizeof total, cudaMemcpyDeviceToHost));
        PT_CUDA(cudaMemcpy(&t0, buf.start_ns, sizeof t0, cudaMemcpyDeviceToHost));
        std::vector<unsigned long long> done(static_cast<size_t>(njobs));
        PT_CUDA(cudaMemcpy(done.data(), buf.job_done_ns, done.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        rays = total;
        job_ms.assign(size_t(njobs), 0.0);
        for (int32_t k = 0; k < njobs; k++) job_ms[size_t(k)] = done[size_t(k)] > t0 ? double(done[size_t(k)] - t0) / 1e6 : 0.0;
    }
};

namespace {
// Merges every scene's host layout into one: four-wide nodes, slots, primitives, materials,
// textures, pixels and emitter tables, with their indices offset.
void merge_scenes(pt_batch *b, const pt_scene_desc *descs, int32_t count, std::vector<int32_t> &roots, std::vector<int32_t> &roots2,
                  std::vector<int32_t> &light_offset, std::vector<int32_t> &light_count, std::vector<float> &light_area) {
    std::vector<HostLayout> layouts(static_cast<size_t>(count));
    int64_t total_tri_slots = 0;
    for (int32_t i = 0; i < count; i++) {
        validate_scene(descs[i]);
        layouts[size_t(i)] = relayout(descs[i]);
        if (descs[i].root >= 0 && layouts[size_t(i)].nodes4.empty())
            throw Error(PT_INVALID_ARGUMENT, "batched scenes must be trees (no shared subtrees)");
        total_tri_slots += int64_t(layouts[size_t(i)].tris.size());
    }
    std::vector<Bvh4Node> nodes4;
    std::vector<BvhNode> nodes2;
    std::vector<TriRecord> tris;
    std::vector<SphereRecord> spheres;
    std::vector<pt_triangle> triangles;
    std::vector<pt_sphere> sphere_src;
    std::vector<pt_material> materials;
    std::vector<pt_texture> textures;
    std::vector<unsigned char> pixels;
    std::vector<pt_light> lights;
    int64_t sphere_slot_base = 0;
    for (int32_t i = 0; i < count; i++) {
        const pt_scene_desc &d = descs[i];
        HostLayout &L = layouts[size_t(i)];
        const int32_t node_base = int32_t(nodes4.size()), node2_base = int32_t(nodes2.size());
        const int64_t tri_slot_base = int64_t(tris.size());
        const int32_t local_tri_slots = int32_t(L.tris.size());
        const int32_t tri_base = int32_t(triangles.size()), sphere_base = int32_t(sphere_src.size());
        const int32_t material_base = int32_t(materials.size()), texture_base = int32_t(textures.size());
        const int64_t pixel_base = int64_t(pixels.size());
        if (total_tri_slots + sphere_slot_base + int64_t(L.spheres.size()) >= (int64_t(1) << 28))
            throw Error(PT_INVALID_ARGUMENT, "batched scenes exceed 2^28 primitives");
        roots.push_back(d.root < 0 ? -1 : node_base);
        roots2.push_back(d.root < 0 ? -1 : node2_base);
        // a two-wide leaf reference is ~slot of one primitive
        auto slot2 = [&](int32_t c) -> int32_t {
            if (c == kEmptyChild) return c;
            if (c >= 0) return c + node2_base;
            const int32_t k = ~c;
            const int64_t g = k < local_tri_slots ? tri_slot_base + k : total_tri_slots + sphere_slot_base + (k - local_tri_slots);
            return ~int32_t(g);
        };
        if (d.root >= 0) {
            for (BvhNode n : L.nodes) {
                n.child0 = slot2(n.child0);
                n.child1 = slot2(n.child1);
                nodes2.push_back(n);
            }
        }
        for (Bvh4Node n : L.nodes4) {
            for (int k = 0; k < 4; k++) {
                int32_t c = n.child[k];
                if (c == kEmptyChild) continue;
                if (c >= 0) { n.child[k] = c + node_base; continue; }
                int32_t v = ~c, first = v >> 3, cnt = v & 7;
                int64_t g = first < local_tri_slots ? tri_slot_base + first : total_tri_slots + sphere_slot_base + (first - local_tri_slots);
                n.child[k] = ~int32_t((g << 3) | cnt);
            }
            nodes4.push_back(n);
        }
        for (TriRecord t : L.tris) { t.id += tri_base; tris.push_back(t); }
        for (SphereRecord sp : L.spheres) { sp.id += sphere_base; spheres.push_back(sp); }
        sphere_slot_base += int64_t(L.spheres.size());
        for (size_t k = 0; k < d.triangle_count; k++) { pt_triangle t = d.triangles[k]; t.material_id += material_base; triangles.push_back(t); }
        for (size_t k = 0; k < d.sphere_count; k++) { pt_sphere sp = d.spheres[k]; sp.material_id += material_base; sphere_src.push_back(sp); }
        for (size_t k = 0; k < d.material_count; k++) {
            pt_material m = d.materials[k];
            if (m.texture_id >= 0) m.texture_id += texture_base;
            materials.push_back(m);
        }
        for (size_t k = 0; k < d.texture_count; k++) {
            pt_texture t = d.textures[k];
            if (t.type == PT_TEX_MAP) t.image_id += texture_base;
            if (t.type == PT_TEX_IMAGE) {
                if (pixel_base + t.byte_offset > INT32_MAX) throw Error(PT_INVALID_ARGUMENT, "batched image storage exceeds 32-bit offsets");
                t.byte_offset += int32_t(pixel_base);
            }
            textures.push_back(t);
        }
        pixels.insert(pixels.end(), d.pixels, d.pixels + d.pixel_bytes);
        float area = 0;
        std::vector<pt_light> own = scene_lights(d, area);
        light_offset.push_back(int32_t(lights.size()));
        light_count.push_back(int32_t(own.size()));
        light_area.push_back(area);
        for (pt_light l : own) { l.primitive += l.type == PT_TRIANGLE ? tri_base : sphere_base; lights.push_back(l); }
    }
    b->total_triangles = triangles.size();
    std::vector<Bvh4QNode> nodes4q;
    for (const Bvh4Node &w : nodes4) nodes4q.push_back(quantize4(w));
    b->nodes4.upload(nodes4q); b->nodes2.upload(nodes2); b->tris.upload(tris); b->spheres.upload(spheres); b->triangles.upload(triangles);
    b->sphere_src.upload(sphere_src); b->materials.upload(materials); b->textures.upload(textures);
    b->pixels.upload(pixels.data(), pixels.size()); b->lights.upload(lights);
    DeviceScene &v = b->view;
    v.nodes = nodes2.empty() ? nullptr : b->nodes2.get<BvhNode>();
    v.nodes4 = nodes4.empty() ? nullptr : b->nodes4.get<Bvh4QNode>();
    v.tris = b->tris.get<TriRecord>(); v.spheres = b->spheres.get<SphereRecord>();
    v.triangles = b->triangles.get<pt_triangle>(); v.sphere_src = b->sphere_src.get<pt_sphere>();
    v.materials = b->materials.get<pt_material>(); v.textures = b->textures.get<pt_texture>();
    v.pixels = b->pixels.get<unsigned char>(); v.lights = b->lights.get<pt_light>();
    v.node_count = int32_t(nodes4.size());
    v.tri_slots = int32_t(tris.size()); v.sphere_slots = int32_t(spheres.size());
    v.light_count = 0; v.light_area = 0;   // per job
    v.empty = nodes4.empty() ? 1 : 0;
    v.root_leaf = 0;
}
} // namespace

extern "C" {

pt_status pt_batch_create(const pt_scene_desc *scenes, int32_t scene_count, const pt_job *jobs, int32_t job_count,
                          uint32_t flags, pt_batch **out) {
    return guard([&]() {
        if (!scenes || !jobs || !out || scene_count <= 0 || job_count <= 0) throw Error(PT_INVALID_ARGUMENT, "invalid batch arguments");
        *out = nullptr;
        for (int32_t k = 0; k < job_count; k++) {
            const pt_job &j = jobs[k];
            if (j.scene < 0 || j.scene >= scene_count) throw Error(PT_INVALID_ARGUMENT, "job refers to a missing scene");
            if (j.width <= 0 || j.height <= 0 || uint64_t(j.width) * uint64_t(j.height) > uint64_t(INT32_MAX))
                throw Error(PT_INVALID_ARGUMENT, "image dimensions exceed supported pixel count");
            if (j.samples <= 0) throw Error(PT_INVALID_ARGUMENT, "invalid accumulated sample count");
            if (j.max_depth < 0 || j.max_depth > 100000) throw Error(PT_INVALID_ARGUMENT, "invalid bounce limit");
        }
        require_device();
        auto b = new pt_batch;
        try {
            std::vector<int32_t> roots, roots2, loff, lcount;
            std::vector<float> larea;
            merge_scenes(b, scenes, scene_count, roots, roots2, loff, lcount, larea);
            int64_t offset = 0;
            for (int32_t k = 0; k < job_count; k++) {
                const pt_job &j = jobs[k];
                BatchJob bj{};
                bj.camera = j.camera; bj.width = j.width; bj.height = j.height; bj.samples = j.samples; bj.max_depth = j.max_depth;
                bj.seed = j.seed; bj.pixel_offset = offset; bj.pixel_count = j.width * j.height;
                bj.root = roots[size_t(j.scene)]; bj.root2 = roots2[size_t(j.scene)]; bj.light_offset = loff[size_t(j.scene)]; bj.light_count = lcount[size_t(j.scene)];
                bj.light_area = larea[size_t(j.scene)];
                offset += bj.pixel_count;
                b->host_jobs.push_back(bj);
            }
            b->total_pixels = offset;
            b->mis = (flags & PT_RENDER_MIS) ? 1 : 0;
            b->jobs.upload(b->host_jobs);
            b->sums.resize(size_t(offset) * 3 * sizeof(float));
            b->rng.resize(size_t(offset) * sizeof(Pcg));
            b->counters.resize(4 * sizeof(int32_t));
            b->fetch.resize(4 * sizeof(unsigned long long));
            b->scalars.resize(8 * sizeof(unsigned long long));
            b->job_remaining.resize(size_t(job_count) * sizeof(int32_t));
            b->job_done_ns.resize(size_t(job_count) * sizeof(unsigned long long));
            b->error.resize(sizeof(int32_t));
            BatchBuffers &f = b->buf;
            f.jobs = b->jobs.get<BatchJob>(); f.job_count = job_count; f.total_pixels = offset; f.mis = b->mis;
            f.sums = b->sums.get<float>(); f.rng = b->rng.get<Pcg>();
            f.counters = b->counters.get<int32_t>(); f.fetch = b->fetch.get<unsigned long long>();
            unsigned long long *sc = b->scalars.get<unsigned long long>();
            f.cursor = sc; f.rays = sc + 1; f.start_ns = sc + 2; f.iterations = sc + 3;
            f.job_remaining = b->job_remaining.get<int32_t>(); f.job_done_ns = b->job_done_ns.get<unsigned long long>();
            f.error = b->error.get<int32_t>();
            b->tail_paths = int32_t(std::max<int64_t>(16384, offset / 64));
            PT_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
            PT_CUDA(cudaStreamCreateWithFlags(&b->shadow_stream, cudaStreamNonBlocking));
            b->allocate_slots();
        } catch (...) { delete b; throw; }
        *out = b;
    });
}

pt_status pt_batch_destroy(pt_batch *b) { delete b; return PT_OK; }

pt_status pt_batch_tuning(pt_batch *b, int32_t path_capacity, int32_t block, int32_t min_active, int32_t tail_paths, int32_t use_graph) {
    return guard([&]() {
        if (!b) throw Error(PT_INVALID_ARGUMENT, "null batch");
        if (path_capacity < 0 || !(block == 64 || block == 128 || block == 256) || min_active < 1 || min_active > 32 || tail_paths < 0)
            throw Error(PT_INVALID_ARGUMENT, "invalid batch tuning");
        bool realloc = path_capacity != b->capacity;
        if (block != b->block || min_active != b->min_active || tail_paths != b->tail_paths || use_graph != b->use_graph) b->drop_graph();
        b->capacity = path_capacity; b->block = block; b->min_active = min_active; b->tail_paths = tail_paths;
        b->use_graph = use_graph ? 1 : 0;
        if (realloc) b->allocate_slots();
    });
}

// Node fetch width of the batch's walks: 1 = four-wide nodes, 0 = the two-wide layout.
pt_status pt_batch_node_width(pt_batch *b, int32_t wide) {
    return guard([&]() {
        if (!b) throw Error(PT_INVALID_ARGUMENT, "null batch");
        if ((wide ? 1 : 0) != b->wide) b->drop_graph();
        b->wide = wide ? 1 : 0;
    });
}

pt_status pt_batch_run(pt_batch *b) {
    return guard([&]() {
        if (!b) throw Error(PT_INVALID_ARGUMENT, "null batch");
        b->run();
    });
}

pt_status pt_batch_get_sums(const pt_batch *b, int32_t job, float *rgb, size_t floats) {
    return guard([&]() {
        if (!b || job < 0 || size_t(job) >= b->host_jobs.size()) throw Error(PT_INVALID_ARGUMENT, "no such job");
        const BatchJob &j = b->host_jobs[size_t(job)];
        if (!rgb || floats < size_t(j.pixel_count) * 3) throw Error(PT_INVALID_ARGUMENT, "sum buffer too small");
        PT_CUDA(cudaMemcpy(rgb, b->buf.sums + 3 * size_t(j.pixel_offset), size_t(j.pixel_count) * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

pt_status pt_batch_stats(const pt_batch *b, float *kernel_ms, uint64_t *rays, double *job_completion_ms, size_t jobs) {
    return guard([&]() {
        if (!b) throw Error(PT_INVALID_ARGUMENT, "null batch");
        if (kernel_ms) *kernel_ms = b->milliseconds;
        if (rays) *rays = b->rays;
        for (size_t k = 0; job_completion_ms && k < jobs && k < b->job_ms.size(); k++) job_completion_ms[k] = b->job_ms[k];
    });
}

// Fault injection for tests, on the host: the n-th autotune probe run from now fails as a timed-out
// run would (n <= 0: none).
pt_status pt_batch_fail_probe(pt_batch *b, int32_t n) {
    return guard([&]() {
        if (!b) throw Error(PT_INVALID_ARGUMENT, "null batch");
        b->probe_fault_countdown = n > 0 ? n : 0;
    });
}

// Autotuner: times probe runs (every job at min(probe_samples, its samples)) over path-pool
// capacity, block size, refill threshold and graph/host loop, then the other node fetch width at
// the fastest of those, keeps the fastest, and caches it per (log2 triangles, log2 pixels) bucket
// in a text file (one "bucket capacity block min_active use_graph node_width ms" line per bucket).
// With a cached entry for the bucket the sweep is skipped.
pt_status pt_batch_autotune(pt_batch *b, int32_t probe_samples, const char *cache_path, int32_t *best) {
    return guard([&]() {
        if (!b || probe_samples <= 0) throw Error(PT_INVALID_ARGUMENT, "invalid autotune arguments");
        int tb = int(std::log2(double(std::max<uint64_t>(1, b->total_triangles))));
        int pb = int(std::log2(double(std::max<int64_t>(1, b->total_pixels))));
        std::string bucket = "tri" + std::to_string(tb) + "_px" + std::to_string(pb);
        int32_t cfg[5] = {0, 256, 16, 1, 1};
        bool cached = false;
        std::vector<std::string> lines;
        if (cache_path) {
            std::ifstream in(cache_path);
            std::string line;
            while (std::getline(in, line)) {
                lines.push_back(line);
                std::istringstream ss(line);
                std::string key;
                int32_t c0, c1, c2, c3, c4;
                if (ss >> key >> c0 >> c1 >> c2 >> c3 >> c4 && key == bucket) {
                    cfg[0] = c0; cfg[1] = c1; cfg[2] = c2; cfg[3] = c3; cfg[4] = c4; cached = true;
                }
            }
        }
        if (!cached) {
            // probe: fewer samples per job; the jobs' own sample counts come back on every path out
            struct Restore {
                pt_batch *b;
                std::vector<BatchJob> saved;
                ~Restore() {
                    b->host_jobs = saved;
                    try { b->jobs.upload(b->host_jobs); } catch (...) {}
                }
            } restore{b, b->host_jobs};
            if (!b->wide) { b->wide = 1; b->drop_graph(); }   // the sweep runs on four-wide nodes
            for (auto &j : b->host_jobs) j.samples = std::min(j.samples, probe_samples);
            b->jobs.upload(b->host_jobs);
            const int32_t caps[] = {1 << 20, 1 << 21, 1 << 22};
            const int32_t blocks[] = {128, 256};
            const int32_t actives[] = {8, 16, 24};
            double best_ms = 1e30;
            std::string failure;
            for (int32_t cap : caps) for (int32_t blk : blocks) for (int32_t act : actives) for (int32_t graph : {1, 0}) {
                pt_status st = pt_batch_tuning(b, cap, blk, act, b->tail_paths, graph);
                if (st != PT_OK) continue;
                try {
                    if (b->probe_fault_countdown > 0 && --b->probe_fault_countdown == 0)
                        throw Error(PT_TIMEOUT, "probe run failed (injected on the host)");
                    b->run();
                } catch (const Error &e) {
                    if (e.status == PT_CUDA_ERROR) throw;   // the context may be lost: stop the sweep
                    failure = e.what();                      // this setting failed: skip it
                    continue;
                }
                if (b->milliseconds < best_ms) { best_ms = b->milliseconds; cfg[0] = cap; cfg[1] = blk; cfg[2] = act; cfg[3] = graph; }
            }
            if (best_ms == 1e30) throw Error(PT_INVALID_ARGUMENT, "every autotune setting failed: " + failure);
            // node fetch width at the best setting: the four-wide nodes against the two-wide layout
            for (int32_t w : {0, 1}) {
                if (w == cfg[4]) continue;
                if (pt_batch_tuning(b, cfg[0], cfg[1], cfg[2], b->tail_paths, cfg[3]) != PT_OK) continue;
                b->wide = w;
                b->drop_graph();
                try { b->run(); } catch (const Error &e) { if (e.status == PT_CUDA_ERROR) throw; continue; }
                if (b->milliseconds < best_ms) { best_ms = b->milliseconds; cfg[4] = w; }
            }
            b->wide = cfg[4];
            b->drop_graph();
            if (cache_path) {
                std::ofstream outf(cache_path, std::ios::app);
                outf << bucket << " " << cfg[0] << " " << cfg[1] << " " << cfg[2] << " " << cfg[3] << " " << cfg[4] << " " << best_ms << "\n";
            }
        }
        pt_status st = pt_batch_tuning(b, cfg[0], cfg[1], cfg[2], b->tail_paths, cfg[3]);
        if (st != PT_OK) throw Error(st, pt_last_error());
        if ((cfg[4] ? 1 : 0) != b->wide) { b->wide = cfg[4] ? 1 : 0; b->drop_graph(); }
        if (best) { best[0] = cfg[0]; best[1] = cfg[1]; best[2] = cfg[2]; best[3] = cfg[3]; best[4] = cfg[4]; }
    });
}

} // extern "C"
