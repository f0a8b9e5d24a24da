// pt_device.h — device memory ownership and launch helpers (CUDA runtime, host side).
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>
#include "pt_host.h"

namespace ptb {

inline void cuda_check(cudaError_t result, const char *what) {
    if(result != cudaSuccess) throw Error(PT_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(result));
}
#define PT_CUDA(call) ::ptb::cuda_check((call), #call)

// Owning device allocation (the library's only allocator).
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t bytes) { resize(bytes); }
    ~DeviceBuffer() { release(); }
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    DeviceBuffer(DeviceBuffer &&o) noexcept : ptr_(o.ptr_), bytes_(o.bytes_) { o.ptr_ = nullptr; o.bytes_ = 0; }
    void resize(size_t bytes) {
        if(bytes == bytes_) return;
        release();
        if(bytes) PT_CUDA(cudaMalloc(&ptr_, bytes));
        bytes_ = bytes;
    }
    void reserve(size_t bytes) { if(bytes > bytes_) resize(bytes); }
    template <class T> void upload(const std::vector<T> &v) {
        resize(v.size() * sizeof(T));
        if(bytes_) PT_CUDA(cudaMemcpy(ptr_, v.data(), bytes_, cudaMemcpyHostToDevice));
    }
    void upload(const void *src, size_t bytes) {
        resize(bytes);
        if(bytes) PT_CUDA(cudaMemcpy(ptr_, src, bytes, cudaMemcpyHostToDevice));
    }
    template <class T = void> T *get() const { return static_cast<T *>(ptr_); }
    size_t bytes() const { return bytes_; }
    void release() { if(ptr_) cudaFree(ptr_); ptr_ = nullptr; bytes_ = 0; }
private:
    void *ptr_ = nullptr;
    size_t bytes_ = 0;
};

class Event {
public:
    Event() { PT_CUDA(cudaEventCreate(&e_)); }
    ~Event() { cudaEventDestroy(e_); }
    Event(const Event &) = delete;
    Event &operator=(const Event &) = delete;
    cudaEvent_t get() const { return e_; }
private:
    cudaEvent_t e_{};
};

void require_device();
int device_sm_count();
// Ray counters per scene: launches further apart than this many may share one counter, so a scene
// takes at most this many persistent-kernel launches in flight at once.
constexpr int kRayCounters = 64;

// Tunables of the traversal kernels (pt_query_tuning and friends; process-wide).  Each field is
// atomic, so a setter racing with launches on other threads is well defined; a launch reads each
// field once.
struct QueryConfig {
    std::atomic<int> persistent{1}, min_active{24}, blocks_per_sm{0}, wide{1}, speculative{1};
    std::atomic<int> order{2};             // 0 never, 1 always, 2 when the walked arrays exceed the L2
};
extern QueryConfig g_query_config;

} // namespace ptb

// The scene handle: everything device-resident that queries and renderers read.
struct pt_scene {
    ptb::DeviceScene view{};
    ptb::DeviceBuffer nodes, nodes4, tris, spheres, triangles, sphere_src, materials, textures, pixels, lights, brute_order;
    std::vector<pt_light> host_lights;
    float light_area = 0;
    int32_t leaf_count = 0;
    size_t triangle_count = 0, sphere_count = 0;
    // host-buffer query workspace (reused between calls)
    ptb::DeviceBuffer work_rays[3], work_tmax[3], work_hits[3], work_stats[3];
    cudaStream_t streams[3] = {nullptr, nullptr, nullptr};
    std::mutex work_mutex;                  // one pt_query_rays call at a time uses the workspace above
    ptb::DeviceBuffer ray_counter;          // per-launch ray counters of the persistent query kernel (a ring)
    std::atomic<unsigned> counter_slot{0};
    cudaMemPool_t order_pool = nullptr;     // stream-ordered scratch of the ray ordering (kept, not released)
    int device = 0;
    size_t l2_bytes = 0;                    // L2 size of the scene's device (the ray ordering's threshold)
    // pt_query_profile: CUDA events recorded around each walk-kernel launch (pairs, a ring)
    std::vector<cudaEvent_t> profile_events;
    size_t profile_next = 0;
    ~pt_scene();
};
