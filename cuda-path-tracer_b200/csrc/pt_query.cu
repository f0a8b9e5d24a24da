// pt_query.cu — scene upload and the ray-query kernels (sm_100a, built with --fmad=false).
//
// Replaces cuda_query_rays / query_rays (src/cuda/cuda_renderer.cu:111-120, 248-260) and the
// device_scene upload (src/cuda/cuda_renderer.cu:36-54).
#include <cub/device/device_radix_sort.cuh>
#include <cfloat>
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include "pt_api_common.h"
#include "pt_device.h"
#include "pt_traverse.h"

using namespace ptb;

namespace ptb {

static thread_local std::string g_last_error;
void set_last_error(const std::string &message) { g_last_error = message; }

void require_device() {
    int count = 0;
    cudaError_t st = cudaGetDeviceCount(&count);
    if(st != cudaSuccess) { cudaGetLastError(); throw Error(PT_NO_DEVICE, std::string("CUDA device unavailable: ") + cudaGetErrorString(st)); }
    if(count < 1) throw Error(PT_NO_DEVICE, "CUDA device unavailable: no CUDA devices");
}

int device_sm_count() {
    int dev = 0, sms = 0;
    PT_CUDA(cudaGetDevice(&dev));
    PT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return sms;
}

constexpr int kQueryBlock = 128;

template <bool kAny, bool kStats>
__global__ void __launch_bounds__(kQueryBlock) query_kernel(DeviceScene s, const pt_ray *__restrict__ rays, size_t count,
                                                            float tmin, const float *__restrict__ tmax,
                                                            pt_hit *__restrict__ hits, pt_ray_stats *__restrict__ stats, int tie) {
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(i >= count) return;
    pt_ray r = rays[i];
    float hi = tmax ? tmax[i] : FLT_MAX;
    HitInfo h;
    uint32_t boxes = 0, prims = 0;
    int error = 0;
    bool hit = traverse<kAny>(s, r, tmin, hi, tie, h, boxes, prims, error);
    int32_t type = PT_BRANCH, id = -1;
    if(hit) hit_ids(s, h.slot, type, id);
    int4 out = make_int4(__float_as_int(hit ? h.t : 0.0f), id, type, error);
    reinterpret_cast<int4 *>(hits)[i] = out;
    if(kStats) { stats[i].boxes = boxes; stats[i].primitives = prims; }
}

// Persistent form: a fixed grid of warps; each warp takes rays from a global counter and,
// between traversal steps, hands a new ray to every lane whose ray has ended once fewer than
// `min_active` lanes are still busy.  next_ray must be zero at launch.
// `order` (may be null) lists the rays in the order they are taken: the k-th ray taken is
// rays[order[k]], and its answer goes to hits[order[k]].
template <bool kAny, bool kStats, int kWalk>
__global__ void __launch_bounds__(kQueryBlock, 8) query_persistent_kernel(DeviceScene s, const pt_ray *__restrict__ rays, size_t count,
                                                                       float tmin, const float *__restrict__ tmax,
                                                                       pt_hit *__restrict__ hits, pt_ray_stats *__restrict__ stats,
                                                                       int tie, unsigned long long *next_ray, int min_active,
                                                                       const uint32_t *__restrict__ order) {
    auto get = [&](size_t k, pt_ray &r, float &lo, float &hi) {
        const size_t i = order ? size_t(order[k]) : k;
        r = rays[i]; lo = tmin; hi = tmax ? tmax[i] : FLT_MAX;
    };
    auto done = [&](size_t k, const WalkResult &w) {
        const size_t i = order ? size_t(order[k]) : k;
        bool hit = w.slot >= 0;
        int32_t type = PT_BRANCH, id = -1;
        if (hit) hit_ids(s, w.slot, type, id);
        reinterpret_cast<int4 *>(hits)[i] = make_int4(__float_as_int(hit ? w.t : 0.0f), id, type, w.error);
        if (kStats) { stats[i].boxes = w.boxes; stats[i].primitives = w.prims; }
    };
    if (kWalk == 2) persistent_walk4_spec<kAny>(s, count, next_ray, min_active, tie, get, done);
    else if (kWalk == 1) persistent_walk4<kAny>(s, count, next_ray, min_active, tie, get, done);
    else persistent_walk<kAny>(s, count, next_ray, min_active, tie, get, done);
}

template <bool kAny, bool kStats>
__global__ void __launch_bounds__(kQueryBlock) brute_kernel(DeviceScene s, const int32_t *__restrict__ order, int32_t leaves,
                                                            const pt_ray *__restrict__ rays, size_t count, float tmin,
                                                            const float *__restrict__ tmax, pt_hit *__restrict__ hits,
                                                            pt_ray_stats *__restrict__ stats, int tie) {
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(i >= count) return;
    pt_ray r = rays[i];
    float hi = tmax ? tmax[i] : FLT_MAX;
    HitInfo h;
    uint32_t prims = 0;
    bool hit = traverse_brute<kAny>(s, order, leaves, r, tmin, hi, tie, h, prims);
    int32_t type = PT_BRANCH, id = -1;
    if(hit) hit_ids(s, h.slot, type, id);
    reinterpret_cast<int4 *>(hits)[i] = make_int4(__float_as_int(hit ? h.t : 0.0f), id, type, 0);
    if(kStats) { stats[i].boxes = 0; stats[i].primitives = prims; }
}

// query_rays (src/cuda/cuda_renderer.cu:111-120): full trace_result, reference tie rule.
__global__ void __launch_bounds__(kQueryBlock) compat_kernel(DeviceScene s, const int32_t *__restrict__ order, int32_t leaves,
                                                             const pt_ray *__restrict__ rays, size_t count, int brute,
                                                             pt_trace_result *__restrict__ out) {
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(i >= count) return;
    pt_ray r = rays[i];
    HitInfo h;
    uint32_t boxes = 0, prims = 0;
    int error = 0;
    bool hit = brute ? traverse_brute<false>(s, order, leaves, r, 0.001f, FLT_MAX, kTieLastNode, h, prims)
                     : traverse<false>(s, r, 0.001f, FLT_MAX, kTieLastLeaf, h, boxes, prims, error);
    pt_trace_result res;
    res.rec.t = 0; res.rec.u = 0; res.rec.v = 0;
    res.rec.p = pt_vec3{0, 0, 0}; res.rec.normal = pt_vec3{0, 0, 0};
    res.rec.material_id = -1; res.rec.primitive_type = -1; res.rec.primitive_id = -1;
    if(hit) finalize_hit(s, r, h, res.rec);
    res.hit = hit ? 1 : 0;
    res.error = error;
    out[i] = res;
}

// Camera rays, one PCG stream per ray (same arithmetic as pt_rays_camera on the host).
__global__ void camera_rays_kernel(pt_camera c, int width, int height, uint64_t seed, uint64_t first, size_t count, pt_ray *rays) {
    size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(k >= count) return;
    uint64_t index = first + k;
    uint64_t pixel = index % (uint64_t(width) * uint64_t(height));
    int x = int(pixel % uint64_t(width)), y = int(pixel / uint64_t(width));
    Pcg r; r.seed(seed, index);
    float u = (x + r.uniform()) / float(width);
    float v = (y + r.uniform()) / float(height);
    pt_ray out;
    camera_ray(c, u, v, r, out);
    rays[k] = out;
}

// Bounce rays: from each primary hit, a cosine-distributed direction about the geometric
// normal turned toward the incoming ray; a primary miss is replaced by a random surface ray.
__global__ void bounce_rays_kernel(DeviceScene s, const pt_ray *primary, const pt_hit *hits, size_t count,
                                   uint64_t seed, uint64_t first, uint64_t triangles, pt_ray *out) {
    size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(k >= count) return;
    pt_ray o;
    bounce_ray(s.triangles, triangles, s.sphere_src, primary[k], hits[k], seed, first + k, o);
    out[k] = o;
}

// Surface rays (same arithmetic as pt_rays_surface on the host).
__global__ void surface_rays_kernel(const pt_triangle *tris, uint64_t triangles, uint64_t seed, uint64_t first, size_t count,
                                    pt_ray *rays, float *tmax) {
    size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if(k >= count) return;
    pt_ray o;
    float hi = 0;
    surface_ray(tris, triangles, seed, first + k, tmax != nullptr, o, &hi);
    rays[k] = o;
    if(tmax) tmax[k] = hi;
}

unsigned grid_for(size_t count, int block) { return unsigned((count + size_t(block) - 1) / size_t(block)); }

// ---- ray ordering -----------------------------------------------------------------------------
// A batch of at least kOrderMin rays is walked in the order of a 30-bit key: the direction's
// octant (3 bits) above a Morton code of the origin in the scene's root box (9 bits per axis).
// Rays that start close together and head the same way then share warps and walk the same nodes:
// fewer idle lanes, more cache hits.  The sort is stable and only changes which lane walks which
// ray, so every answer is the same.
constexpr size_t kOrderMin = size_t(1) << 18;
constexpr int kOrderBits = 30;

__device__ inline uint32_t spread_bits3(uint32_t v) {   // 9 bits -> every third bit of 27
    v &= 0x1ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void ray_keys_kernel(const pt_ray *__restrict__ rays, size_t count, float3 lo, float3 scale, uint32_t *__restrict__ keys,
                                uint32_t *__restrict__ index) {
    size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const pt_ray r = rays[k];
    // fmaxf(NaN, 0) is 0: a non-finite origin still gets a key
    uint32_t x = uint32_t(fminf(fmaxf((r.origin.x - lo.x) * scale.x, 0.0f), 511.0f));
    uint32_t y = uint32_t(fminf(fmaxf((r.origin.y - lo.y) * scale.y, 0.0f), 511.0f));
    uint32_t z = uint32_t(fminf(fmaxf((r.origin.z - lo.z) * scale.z, 0.0f), 511.0f));
    uint32_t octant = (r.direction.x < 0.0f ? 1u : 0u) | (r.direction.y < 0.0f ? 2u : 0u) | (r.direction.z < 0.0f ? 4u : 0u);
    keys[k] = (octant << 27) | spread_bits3(x) | (spread_bits3(y) << 1) | (spread_bits3(z) << 2);
    index[k] = uint32_t(k);
}

// Sorts the batch's ray indices by key into scratch from the scene's memory pool (allocated and
// freed in stream order, so concurrent queries on other streams get their own).  Returns the
// order and the scratch to free after the walk.
// Ordering pays when the walked arrays do not fit in L2 (the walk is then bound by its node and
// triangle fetches); with an L2-resident tree the sort costs more than it saves.
bool walks_ordered(const pt_scene *sc, bool wide, size_t count) {
    const size_t walk_bytes = (wide ? sc->nodes4.bytes() : sc->nodes.bytes()) + sc->tris.bytes() + sc->spheres.bytes();
    const int mode = g_query_config.order;
    const bool ordered = mode == 1 || (mode == 2 && walk_bytes > sc->l2_bytes);
    return ordered && count >= kOrderMin && count <= size_t(INT32_MAX) && sc->order_pool;
}

const uint32_t *order_rays(const pt_scene *sc, const pt_ray *rays, size_t count, cudaStream_t stream, void *&scratch) {
    const DeviceScene &s = sc->view;
    float3 lo = make_float3(s.root_lo[0], s.root_lo[1], s.root_lo[2]);
    float3 scale;
    float ext[3] = {s.root_hi[0] - s.root_lo[0], s.root_hi[1] - s.root_lo[1], s.root_hi[2] - s.root_lo[2]};
    scale.x = ext[0] > 0 ? 512.0f / ext[0] : 0.0f;
    scale.y = ext[1] > 0 ? 512.0f / ext[1] : 0.0f;
    scale.z = ext[2] > 0 ? 512.0f / ext[2] : 0.0f;
    const int n = int(count);
    size_t temp = 0;
    PT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                            (const uint32_t *)nullptr, (uint32_t *)nullptr, n, 0, kOrderBits, stream));
    const size_t words = (count + 63) & ~size_t(63);          // 256-byte aligned sub-arrays
    const size_t bytes = 4 * words * sizeof(uint32_t) + temp;
    PT_CUDA(cudaMallocFromPoolAsync(&scratch, bytes, sc->order_pool, stream));
    uint32_t *keys_in = static_cast<uint32_t *>(scratch), *keys_out = keys_in + words;
    uint32_t *index_in = keys_out + words, *index_out = index_in + words;
    void *temp_storage = index_out + words;
    ray_keys_kernel<<<grid_for(count, 256), 256, 0, stream>>>(rays, count, lo, scale, keys_in, index_in);
    PT_CUDA(cudaGetLastError());
    PT_CUDA(cub::DeviceRadixSort::SortPairs(temp_storage, temp, keys_in, keys_out, index_in, index_out, n, 0, kOrderBits, stream));
    return index_out;
}

// Query kernel variant and its tunables (the autotuner sets these).
QueryConfig g_query_config;

// Resident blocks per SM of query-kernel variant `k` on `device` (the occupancy calculator's
// answer, looked up once per device and variant).
int blocks_per_sm(int device, int k, const void *fn, size_t smem) {
    static std::mutex mutex;
    static std::map<std::pair<int, int>, int> cache;
    std::lock_guard<std::mutex> lock(mutex);
    auto it = cache.find({device, k});
    if (it != cache.end()) return it->second;
    int n = 0;
    PT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kQueryBlock, smem));
    cache[{device, k}] = n;
    return n;
}

void launch_query(const pt_scene *sc, const pt_ray *rays, size_t count, int mode, float tmin, const float *tmax,
                  pt_hit *hits, pt_ray_stats *stats, int tie, cudaStream_t stream) {
    if(!count) return;
    const DeviceScene &s = sc->view;
    if(g_query_config.persistent) {
        pt_scene *m = const_cast<pt_scene *>(sc);
        unsigned long long *counter = m->ray_counter.get<unsigned long long>() + (m->counter_slot.fetch_add(1) % kRayCounters);
        PT_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream));
        const bool wide = g_query_config.wide && s.nodes4;
        const bool any = mode == PT_QUERY_ANY;
        using Fn = void (*)(DeviceScene, const pt_ray *, size_t, float, const float *, pt_hit *, pt_ray_stats *, int,
                            unsigned long long *, int, const uint32_t *);
        static const Fn table[12] = {
            query_persistent_kernel<false, false, 0>, query_persistent_kernel<false, false, 1>, query_persistent_kernel<false, false, 2>,
            query_persistent_kernel<false, true, 0>, query_persistent_kernel<false, true, 1>, query_persistent_kernel<false, true, 2>,
            query_persistent_kernel<true, false, 0>, query_persistent_kernel<true, false, 1>, query_persistent_kernel<true, false, 2>,
            query_persistent_kernel<true, true, 0>, query_persistent_kernel<true, true, 1>, query_persistent_kernel<true, true, 2>};
        int walk = wide ? (g_query_config.speculative ? 2 : 1) : 0;
        int k = (any ? 6 : 0) + (stats ? 3 : 0) + walk;
        Fn fn = table[k];
        const size_t smem = wide ? size_t(kSharedStack4) * kQueryBlock * sizeof(int2) : size_t(kSharedStack) * kQueryBlock * sizeof(int32_t);
        const int occupancy = blocks_per_sm(sc->device, k, (const void *)fn, smem);
        const int want_bps = g_query_config.blocks_per_sm;
        int bps = want_bps > 0 ? std::min(want_bps, occupancy) : occupancy;
        size_t want = (count + kQueryBlock - 1) / kQueryBlock;
        unsigned grid = unsigned(std::min<size_t>(want, size_t(device_sm_count()) * size_t(bps > 0 ? bps : 1)));
        void *scratch = nullptr;
        const uint32_t *order = nullptr;
        if (walks_ordered(sc, wide, count)) {
            cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
            PT_CUDA(cudaStreamIsCapturing(stream, &capture));
            if (capture == cudaStreamCaptureStatusNone) order = order_rays(sc, rays, count, stream, scratch);   // not inside a graph capture
        }
        cudaEvent_t *ev = nullptr;
        if (!m->profile_events.empty()) {
            const size_t pairs = m->profile_events.size() / 2;
            ev = &m->profile_events[2 * (m->profile_next++ % pairs)];
            PT_CUDA(cudaEventRecord(ev[0], stream));
        }
        fn<<<grid, kQueryBlock, smem, stream>>>(s, rays, count, tmin, tmax, hits, stats, tie, counter, g_query_config.min_active,
                                                 order);
        PT_CUDA(cudaGetLastError());
        if (ev) PT_CUDA(cudaEventRecord(ev[1], stream));
        if (scratch) PT_CUDA(cudaFreeAsync(scratch, stream));
        return;
    }
    unsigned grid = grid_for(count, kQueryBlock);
    if(mode == PT_QUERY_ANY) {
        if(stats) query_kernel<true, true><<<grid, kQueryBlock, 0, stream>>>(s, rays, count, tmin, tmax, hits, stats, tie);
        else query_kernel<true, false><<<grid, kQueryBlock, 0, stream>>>(s, rays, count, tmin, tmax, hits, stats, tie);
    } else {
        if(stats) query_kernel<false, true><<<grid, kQueryBlock, 0, stream>>>(s, rays, count, tmin, tmax, hits, stats, tie);
        else query_kernel<false, false><<<grid, kQueryBlock, 0, stream>>>(s, rays, count, tmin, tmax, hits, stats, tie);
    }
    PT_CUDA(cudaGetLastError());
}

} // namespace ptb

pt_scene::~pt_scene() {
    for(auto &e : profile_events) cudaEventDestroy(e);
    for(auto &s : streams) if(s) cudaStreamDestroy(s);
    // a pool destroyed with frees still pending on a stream is released once they complete
    if(order_pool) cudaMemPoolDestroy(order_pool);
}

extern "C" {

const char *pt_last_error(void) { return g_last_error.c_str(); }
int pt_abi_version(void) { return PT_ABI_VERSION; }

// cuda_device_available, src/cuda/cuda_renderer.cu:128-140
int pt_device_available(char *description, size_t capacity) {
    std::string text;
    int ok = 0;
    int count = 0;
    cudaError_t status = cudaGetDeviceCount(&count);
    if(status != cudaSuccess) { text = cudaGetErrorString(status); cudaGetLastError(); }
    else if(count < 1) text = "no CUDA devices";
    else {
        int current = 0;
        cudaDeviceProp properties{};
        status = cudaGetDevice(&current);
        if(status == cudaSuccess) status = cudaGetDeviceProperties(&properties, current);
        if(status != cudaSuccess) text = cudaGetErrorString(status);
        else { text = properties.name; ok = 1; }
    }
    if(description && capacity) {
        std::strncpy(description, text.c_str(), capacity - 1);
        description[capacity - 1] = 0;
    }
    return ok;
}

pt_status pt_scene_create(const pt_scene_desc *desc, pt_scene **out) {
    return guard([&]() {
        if(!desc || !out) throw Error(PT_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        validate_scene(*desc);
        require_device();
        float area = 0;
        std::vector<pt_light> lights = scene_lights(*desc, area);
        HostLayout layout = relayout(*desc);
        auto sc = new pt_scene;
        try {
            PT_CUDA(cudaGetDevice(&sc->device));
            {
                int l2 = 0;
                PT_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, sc->device));
                sc->l2_bytes = size_t(l2 > 0 ? l2 : 0);
            }
            {   // the ray ordering's scratch pool: memory stays with the pool between queries
                cudaMemPoolProps props{};
                props.allocType = cudaMemAllocationTypePinned;
                props.location.type = cudaMemLocationTypeDevice;
                props.location.id = sc->device;
                PT_CUDA(cudaMemPoolCreate(&sc->order_pool, &props));
                uint64_t keep = UINT64_MAX;
                PT_CUDA(cudaMemPoolSetAttribute(sc->order_pool, cudaMemPoolAttrReleaseThreshold, &keep));
            }
            sc->ray_counter.resize(sizeof(unsigned long long) * kRayCounters);
            sc->host_lights = lights;
            sc->light_area = area;
            sc->triangle_count = desc->triangle_count;
            sc->sphere_count = desc->sphere_count;
            sc->nodes.upload(layout.nodes);
            sc->nodes4.upload(layout.nodes4q);
            sc->tris.upload(layout.tris);
            sc->spheres.upload(layout.spheres);
            sc->brute_order.upload(layout.brute_order);
            sc->triangles.upload(desc->triangles, desc->triangle_count * sizeof(pt_triangle));
            sc->sphere_src.upload(desc->spheres, desc->sphere_count * sizeof(pt_sphere));
            sc->materials.upload(desc->materials, desc->material_count * sizeof(pt_material));
            sc->textures.upload(desc->textures, desc->texture_count * sizeof(pt_texture));
            sc->pixels.upload(desc->pixels, desc->pixel_bytes);
            sc->lights.upload(lights);
            sc->leaf_count = int32_t(layout.brute_order.size());
            DeviceScene &v = sc->view;
            v.nodes = sc->nodes.get<BvhNode>();
            v.nodes4 = layout.nodes4q.empty() ? nullptr : sc->nodes4.get<Bvh4QNode>();
            v.tris = sc->tris.get<TriRecord>();
            v.spheres = sc->spheres.get<SphereRecord>();
            v.triangles = sc->triangles.get<pt_triangle>();
            v.sphere_src = sc->sphere_src.get<pt_sphere>();
            v.materials = sc->materials.get<pt_material>();
            v.textures = sc->textures.get<pt_texture>();
            v.pixels = sc->pixels.get<unsigned char>();
            v.lights = sc->lights.get<pt_light>();
            v.node_count = int32_t(layout.nodes.size());
            v.tri_slots = int32_t(layout.tris.size());
            v.sphere_slots = int32_t(layout.spheres.size());
            v.light_count = int32_t(lights.size());
            v.light_area = area;
            v.empty = layout.empty;
            for(int a = 0; a < 3; a++) { v.root_lo[a] = layout.root_lo[a]; v.root_hi[a] = layout.root_hi[a]; }
            v.root_leaf = layout.root_leaf;
        } catch(...) { delete sc; throw; }
        *out = sc;
    });
}

pt_status pt_scene_destroy(pt_scene *scene) { delete scene; return PT_OK; }

pt_status pt_scene_lights(const pt_scene *scene, pt_light *lights, size_t capacity, size_t *count, float *total_area) {
    return guard([&]() {
        if(!scene) throw Error(PT_INVALID_ARGUMENT, "null scene");
        if(count) *count = scene->host_lights.size();
        if(total_area) *total_area = scene->light_area;
        for(size_t i = 0; i < capacity && i < scene->host_lights.size(); i++) lights[i] = scene->host_lights[i];
    });
}

pt_status pt_query_ordered(const pt_scene *s, size_t count, int *ordered) {
    return guard([&]() {
        if(!s || !ordered) throw Error(PT_INVALID_ARGUMENT, "null argument");
        const bool wide = g_query_config.wide && s->view.nodes4;
        *ordered = g_query_config.persistent && walks_ordered(s, wide, count) ? 1 : 0;
    });
}

pt_status pt_scene_device_bytes(const pt_scene *s, size_t *bytes) {
    return guard([&]() {
        if(!s || !bytes) throw Error(PT_INVALID_ARGUMENT, "null argument");
        *bytes = s->nodes.bytes() + s->nodes4.bytes() + s->tris.bytes() + s->spheres.bytes() + s->triangles.bytes() + s->sphere_src.bytes() +
                 s->materials.bytes() + s->textures.bytes() + s->pixels.bytes() + s->lights.bytes() + s->brute_order.bytes();
    });
}

pt_status pt_query_rays_device(const pt_scene *scene, const pt_ray *rays, size_t count, int mode, float tmin,
                               const float *tmax, pt_hit *hits, pt_ray_stats *stats, void *stream) {
    return guard([&]() {
        if(!scene || (count && (!rays || !hits))) throw Error(PT_INVALID_ARGUMENT, "null argument");
        if(mode != PT_QUERY_CLOSEST && mode != PT_QUERY_ANY) throw Error(PT_INVALID_ARGUMENT, "unknown query mode");
        launch_query(scene, rays, count, mode, tmin, tmax, hits, stats, kTieLowestId, static_cast<cudaStream_t>(stream));
    });
}

// Brute-force form (every leaf, node-array order); used for parity checks.
pt_status pt_query_rays_brute_device(const pt_scene *scene, const pt_ray *rays, size_t count, int mode, float tmin,
                                     const float *tmax, pt_hit *hits, pt_ray_stats *stats, void *stream) {
    return guard([&]() {
        if(!scene || (count && (!rays || !hits))) throw Error(PT_INVALID_ARGUMENT, "null argument");
        if(!count) return;
        unsigned grid = grid_for(count, kQueryBlock);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const int32_t *order = scene->brute_order.get<int32_t>();
        if(mode == PT_QUERY_ANY) {
            if(stats) brute_kernel<true, true><<<grid, kQueryBlock, 0, st>>>(scene->view, order, scene->leaf_count, rays, count, tmin, tmax, hits, stats, kTieLowestId);
            else brute_kernel<true, false><<<grid, kQueryBlock, 0, st>>>(scene->view, order, scene->leaf_count, rays, count, tmin, tmax, hits, stats, kTieLowestId);
        } else {
            if(stats) brute_kernel<false, true><<<grid, kQueryBlock, 0, st>>>(scene->view, order, scene->leaf_count, rays, count, tmin, tmax, hits, stats, kTieLowestId);
            else brute_kernel<false, false><<<grid, kQueryBlock, 0, st>>>(scene->view, order, scene->leaf_count, rays, count, tmin, tmax, hits, stats, kTieLowestId);
        }
        PT_CUDA(cudaGetLastError());
    });
}

// Host buffers: chunks of rays flow through three streams so the upload of one chunk, the
// traversal of the next and the download of a third overlap.
pt_status pt_query_rays(const pt_scene *cscene, const pt_ray *rays, size_t count, int mode, float tmin,
                        const float *tmax, pt_hit *hits, pt_ray_stats *stats) {
    return guard([&]() {
        pt_scene *scene = const_cast<pt_scene *>(cscene);
        if(!scene || (count && (!rays || !hits))) throw Error(PT_INVALID_ARGUMENT, "null argument");
        if(mode != PT_QUERY_CLOSEST && mode != PT_QUERY_ANY) throw Error(PT_INVALID_ARGUMENT, "unknown query mode");
        if(!count) return;
        std::lock_guard<std::mutex> lock(scene->work_mutex);   // the staging buffers are the scene's
        // chunks of 2^20 rays (29 MB in, 17 MB out) over three streams: copies in, walk, copies out
        // overlap, and the unhidden first upload and last download stay short (2^22: 21.5 ms for
        // 2^25 rays, 2^20: 19.8-20.7 ms, against 18.6 ms for the bare copies both ways at once)
        const size_t chunk = size_t(1) << 20;
        size_t per = count < chunk ? count : chunk;
        for(int k = 0; k < 3; k++) {
            if(!scene->streams[k]) PT_CUDA(cudaStreamCreateWithFlags(&scene->streams[k], cudaStreamNonBlocking));
            scene->work_rays[k].reserve(per * sizeof(pt_ray));
            scene->work_hits[k].reserve(per * sizeof(pt_hit));
            if(tmax) scene->work_tmax[k].reserve(per * sizeof(float));
            if(stats) scene->work_stats[k].reserve(per * sizeof(pt_ray_stats));
        }
        size_t chunks = (count + chunk - 1) / chunk;
        for(size_t c = 0; c < chunks; c++) {
            int k = int(c % 3);
            cudaStream_t st = scene->streams[k];
            size_t b = c * chunk, n = count - b < chunk ? count - b : chunk;
            PT_CUDA(cudaMemcpyAsync(scene->work_rays[k].get(), rays + b, n * sizeof(pt_ray), cudaMemcpyHostToDevice, st));
            if(tmax) PT_CUDA(cudaMemcpyAsync(scene->work_tmax[k].get(), tmax + b, n * sizeof(float), cudaMemcpyHostToDevice, st));
            launch_query(scene, scene->work_rays[k].get<pt_ray>(), n, mode, tmin, tmax ? scene->work_tmax[k].get<float>() : nullptr,
                         scene->work_hits[k].get<pt_hit>(), stats ? scene->work_stats[k].get<pt_ray_stats>() : nullptr,
                         kTieLowestId, st);
            PT_CUDA(cudaMemcpyAsync(hits + b, scene->work_hits[k].get(), n * sizeof(pt_hit), cudaMemcpyDeviceToHost, st));
            if(stats) PT_CUDA(cudaMemcpyAsync(stats + b, scene->work_stats[k].get(), n * sizeof(pt_ray_stats), cudaMemcpyDeviceToHost, st));
        }
        for(int k = 0; k < 3; k++) PT_CUDA(cudaStreamSynchronize(scene->streams[k]));
    });
}

pt_status pt_query_rays_compat(const pt_scene *scene, const pt_ray *rays, size_t count, int brute, pt_trace_result *results) {
    return guard([&]() {
        if(!scene || (count && (!rays || !results))) throw Error(PT_INVALID_ARGUMENT, "null argument");
        if(!count) return;
        if(count > size_t(INT32_MAX)) throw Error(PT_INVALID_ARGUMENT, "too many validation rays");
        DeviceBuffer in(count * sizeof(pt_ray)), out(count * sizeof(pt_trace_result));
        PT_CUDA(cudaMemcpy(in.get(), rays, count * sizeof(pt_ray), cudaMemcpyHostToDevice));
        compat_kernel<<<grid_for(count, kQueryBlock), kQueryBlock>>>(scene->view, scene->brute_order.get<int32_t>(), scene->leaf_count,
                                                                     in.get<pt_ray>(), count, brute, out.get<pt_trace_result>());
        PT_CUDA(cudaGetLastError());
        PT_CUDA(cudaDeviceSynchronize());
        PT_CUDA(cudaMemcpy(results, out.get(), count * sizeof(pt_trace_result), cudaMemcpyDeviceToHost));
    });
}

// Query-kernel tuning knobs: persistent (1) or one-thread-per-ray (0) launch, the busy-lane
// count below which a persistent warp refills, and blocks per SM (0 = occupancy limit).
pt_status pt_query_tuning(int persistent, int min_active, int blocks_per_sm) {
    return guard([&]() {
        if(min_active < 1 || min_active > 32 || blocks_per_sm < 0) throw Error(PT_INVALID_ARGUMENT, "invalid query tuning");
        g_query_config.persistent = persistent ? 1 : 0;
        g_query_config.min_active = min_active;
        g_query_config.blocks_per_sm = blocks_per_sm;
    });
}

// Node layout of the traversal kernels: 1 = four-wide nodes where the scene has them, 0 = two-wide.
pt_status pt_query_layout(int wide) {
    return guard([&]() { g_query_config.wide = wide ? 1 : 0; });
}

// Four-wide walk form: 1 = node and leaf phases (speculative while-while), 0 = one loop.
pt_status pt_query_walk(int speculative) {
    return guard([&]() { g_query_config.speculative = speculative ? 1 : 0; });
}

// Ray ordering of large batches: 1 = walk rays in (octant, origin Morton code) order, 0 = as given,
// 2 = ordered only when the scene's walked arrays exceed the device's L2.
pt_status pt_query_order(int mode) {
    return guard([&]() {
        if (mode < 0 || mode > 2) throw Error(PT_INVALID_ARGUMENT, "ray ordering mode must be 0, 1 or 2");
        g_query_config.order = mode;
    });
}

// Walk-kernel timing: `launches` > 0 creates that many event pairs (recorded around each later
// walk-kernel launch of this scene, a ring); 0 removes them.
pt_status pt_query_profile(pt_scene *scene, int launches) {
    return guard([&]() {
        if(!scene || launches < 0) throw Error(PT_INVALID_ARGUMENT, "invalid profile arguments");
        PT_CUDA(cudaDeviceSynchronize());
        for(auto &e : scene->profile_events) cudaEventDestroy(e);
        scene->profile_events.clear();
        scene->profile_next = 0;
        for(int k = 0; k < 2 * launches; k++) {
            cudaEvent_t e;
            PT_CUDA(cudaEventCreate(&e));
            scene->profile_events.push_back(e);
        }
    });
}

// Durations (ms) of the walk launches recorded since pt_query_profile, oldest first (at most the
// ring's size); waits for the last one.
pt_status pt_query_profile_read(pt_scene *scene, float *ms, size_t capacity, size_t *count) {
    return guard([&]() {
        if(!scene || !count) throw Error(PT_INVALID_ARGUMENT, "null argument");
        const size_t pairs = scene->profile_events.size() / 2;
        const size_t n = std::min(scene->profile_next, pairs);
        *count = n;
        for(size_t k = 0; k < n && k < capacity; k++) {
            size_t slot = (scene->profile_next - n + k) % pairs;
            PT_CUDA(cudaEventSynchronize(scene->profile_events[2 * slot + 1]));
            PT_CUDA(cudaEventElapsedTime(&ms[k], scene->profile_events[2 * slot], scene->profile_events[2 * slot + 1]));
        }
    });
}

// ---- no-allocation query ---------------------------------------------------------------------
// Scratch of pt_query_rays_static, shared by every call on a device: the persistent kernel's
// ray counter, then staging for PT_STATIC_QUERY_MAX_RAYS rays, tmax values, hits and counters.
namespace {
constexpr size_t kStaticRays = PT_STATIC_QUERY_MAX_RAYS;
constexpr size_t kStaticRaysOffset = 256;
constexpr size_t kStaticTmaxOffset = kStaticRaysOffset + kStaticRays * sizeof(pt_ray);
constexpr size_t kStaticHitsOffset = kStaticTmaxOffset + kStaticRays * sizeof(float);
constexpr size_t kStaticStatsOffset = kStaticHitsOffset + kStaticRays * sizeof(pt_hit);
constexpr size_t kStaticScratchBytes = kStaticStatsOffset + kStaticRays * sizeof(pt_ray_stats);
static_assert(kStaticHitsOffset % 16 == 0 && kStaticStatsOffset % 8 == 0, "scratch alignment");
}

static __device__ __align__(256) unsigned char g_static_query_scratch[kStaticScratchBytes];

namespace {
// Device address of g_static_query_scratch, looked up once per device with that device current.
std::mutex g_static_mutex;
unsigned char *g_static_address[64] = {nullptr};

unsigned char *static_scratch() {
    int dev = 0;
    PT_CUDA(cudaGetDevice(&dev));
    if(dev < 0 || dev >= 64) throw Error(PT_INVALID_ARGUMENT, "device index beyond 63");
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if(!g_static_address[dev]) {
        void *ptr = nullptr;
        cudaError_t st = cudaGetSymbolAddress(&ptr, g_static_query_scratch);
        if(st != cudaSuccess) throw Error(PT_CUDA_ERROR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(st));
        g_static_address[dev] = static_cast<unsigned char *>(ptr);
    }
    return g_static_address[dev];
}
} // namespace

// Callers that cannot let a library allocate device memory get this form of pt_query_rays: no
// cudaMalloc or cudaFree, no streams or events created; it stages through the static array above.
pt_status pt_query_rays_static(const pt_scene *scene, const pt_ray *rays, size_t count, int mode, float tmin,
                               const float *tmax, pt_hit *hits, pt_ray_stats *stats, void *stream) {
    return guard([&]() {
        if(!scene || (count && (!rays || !hits))) throw Error(PT_INVALID_ARGUMENT, "null argument");
        if(mode != PT_QUERY_CLOSEST && mode != PT_QUERY_ANY) throw Error(PT_INVALID_ARGUMENT, "unknown query mode");
        if(count > kStaticRays)
            throw Error(PT_INVALID_ARGUMENT, "pt_query_rays_static takes at most " + std::to_string(kStaticRays) +
                                                 " rays per call (its static scratch); got " + std::to_string(count));
        if(!count) return;
        unsigned char *base = static_scratch();
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        unsigned long long *counter = reinterpret_cast<unsigned long long *>(base);
        pt_ray *d_rays = reinterpret_cast<pt_ray *>(base + kStaticRaysOffset);
        float *d_tmax = tmax ? reinterpret_cast<float *>(base + kStaticTmaxOffset) : nullptr;
        pt_hit *d_hits = reinterpret_cast<pt_hit *>(base + kStaticHitsOffset);
        pt_ray_stats *d_stats = stats ? reinterpret_cast<pt_ray_stats *>(base + kStaticStatsOffset) : nullptr;
        PT_CUDA(cudaMemcpyAsync(d_rays, rays, count * sizeof(pt_ray), cudaMemcpyHostToDevice, st));
        if(tmax) PT_CUDA(cudaMemcpyAsync(d_tmax, tmax, count * sizeof(float), cudaMemcpyHostToDevice, st));
        PT_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));   // the counter must start at zero
        const DeviceScene &s = scene->view;
        const bool wide = g_query_config.wide && s.nodes4 != nullptr;
        const bool any = mode == PT_QUERY_ANY;
        const int walk = wide ? (g_query_config.speculative ? 2 : 1) : 0;
        using Fn = void (*)(DeviceScene, const pt_ray *, size_t, float, const float *, pt_hit *, pt_ray_stats *, int,
                            unsigned long long *, int, const uint32_t *);
        static const Fn table[12] = {
            query_persistent_kernel<false, false, 0>, query_persistent_kernel<false, false, 1>, query_persistent_kernel<false, false, 2>,
            query_persistent_kernel<false, true, 0>, query_persistent_kernel<false, true, 1>, query_persistent_kernel<false, true, 2>,
            query_persistent_kernel<true, false, 0>, query_persistent_kernel<true, false, 1>, query_persistent_kernel<true, false, 2>,
            query_persistent_kernel<true, true, 0>, query_persistent_kernel<true, true, 1>, query_persistent_kernel<true, true, 2>};
        const int k = (any ? 6 : 0) + (stats ? 3 : 0) + walk;
        Fn fn = table[k];
        const size_t smem = wide ? size_t(kSharedStack4) * kQueryBlock * sizeof(int2) : size_t(kSharedStack) * kQueryBlock * sizeof(int32_t);
        int dev = 0;
        PT_CUDA(cudaGetDevice(&dev));
        const int per_sm = blocks_per_sm(dev, k, (const void *)fn, smem);
        size_t want = (count + kQueryBlock - 1) / kQueryBlock;
        unsigned grid = unsigned(std::min<size_t>(want, size_t(device_sm_count()) * size_t(per_sm > 0 ? per_sm : 1)));
        fn<<<grid, kQueryBlock, smem, st>>>(s, d_rays, count, tmin, d_tmax, d_hits, d_stats, kTieLowestId, counter,
                                            g_query_config.min_active, nullptr);
        PT_CUDA(cudaGetLastError());
        PT_CUDA(cudaMemcpyAsync(hits, d_hits, count * sizeof(pt_hit), cudaMemcpyDeviceToHost, st));
        if(stats) PT_CUDA(cudaMemcpyAsync(stats, d_stats, count * sizeof(pt_ray_stats), cudaMemcpyDeviceToHost, st));
        PT_CUDA(cudaStreamSynchronize(st));
    });
}

pt_status pt_rays_camera_device(const pt_camera *camera, int width, int height, uint64_t seed, uint64_t first,
                                size_t count, pt_ray *rays, void *stream) {
    return guard([&]() {
        if(!camera || (count && !rays) || width <= 0 || height <= 0) throw Error(PT_INVALID_ARGUMENT, "invalid camera ray arguments");
        if(!count) return;
        camera_rays_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(*camera, width, height, seed, first, count, rays);
        PT_CUDA(cudaGetLastError());
    });
}

pt_status pt_rays_bounce_device(const pt_scene *scene, const pt_ray *primary, const pt_hit *hits, size_t count,
                                uint64_t seed, uint64_t first, pt_ray *out, void *stream) {
    return guard([&]() {
        if(!scene || (count && (!primary || !hits || !out))) throw Error(PT_INVALID_ARGUMENT, "null argument");
        if(!count) return;
        if(!scene->triangle_count) throw Error(PT_INVALID_ARGUMENT, "bounce rays need triangles");
        bounce_rays_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(scene->view, primary, hits, count, seed,
                                                                                                 first, scene->triangle_count, out);
        PT_CUDA(cudaGetLastError());
    });
}

pt_status pt_rays_surface_device(const pt_scene *scene, uint64_t seed, uint64_t first, size_t count, pt_ray *rays,
                                 float *shadow_tmax, void *stream) {
    return guard([&]() {
        if(!scene || (count && !rays)) throw Error(PT_INVALID_ARGUMENT, "null argument");
        if(!count) return;
        if(!scene->triangle_count) throw Error(PT_INVALID_ARGUMENT, "surface rays need triangles");
        surface_rays_kernel<<<grid_for(count, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            scene->view.triangles, scene->triangle_count, seed, first, count, rays, shadow_tmax);
        PT_CUDA(cudaGetLastError());
    });
}

} // extern "C"
