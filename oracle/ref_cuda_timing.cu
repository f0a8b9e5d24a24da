// ref_cuda_timing.cu — device timing of the reference's own query kernel (BASELINE INFRASTRUCTURE ONLY).
//
// oracle/Makefile compiles this file, for sm_100a with the reference's --fmad=false, into
// oracle/_ref/libref_cuda_timing.so.  It includes the reference's src/cuda/cuda_renderer.cu where
// it lies, so the reference's query_rays kernel, device_scene and device_buffer (file-local in
// that source) are visible here: the scene is uploaded by the reference's own device_scene and
// query_rays (src/cuda/cuda_renderer.cu:111-120) is launched exactly as cuda_query_rays launches it
// (src/cuda/cuda_renderer.cu:248-260: 256 threads per block, tmin 0.001, tmax FLT_MAX), with CUDA
// events around the kernel alone.  Nothing of the reference is restated or changed.
#include "cuda/cuda_renderer.cu"
#include <cstring>
#include "../include/pt.h"

namespace {
flat_scene timing_scene(const pt_scene_desc *d) {
    flat_scene s;
    auto tri = reinterpret_cast<const flat_triangle *>(d->triangles);
    auto sph = reinterpret_cast<const flat_sphere *>(d->spheres);
    auto nod = reinterpret_cast<const flat_node *>(d->nodes);
    auto mat = reinterpret_cast<const flat_material *>(d->materials);
    auto tex = reinterpret_cast<const flat_texture *>(d->textures);
    s.triangles.assign(tri, tri + d->triangle_count);
    s.spheres.assign(sph, sph + d->sphere_count);
    s.nodes.assign(nod, nod + d->node_count);
    s.materials.assign(mat, mat + d->material_count);
    s.textures.assign(tex, tex + d->texture_count);
    s.pixels.assign(d->pixels, d->pixels + d->pixel_bytes);
    s.root = d->root;
    s.max_depth = d->max_depth;
    return s;
}
thread_local std::string timing_error;
}

extern "C" {

const char *reftime_last_error() { return timing_error.c_str(); }

// Uploads the scene with the reference's device_scene, then runs query_rays over `count` rays that
// are already in device memory (`device_rays`, the reference's 28-byte ray layout) `warmup` + `reps`
// times; *kernel_ms = mean device time of one launch (CUDA events around the launch only).  The
// first `sample` results of the last launch are copied to `sample_out` (may be NULL).
int reftime_query(const pt_scene_desc *d, const pt_ray *device_rays, size_t count, int warmup, int reps,
                  float *kernel_ms, pt_trace_result *sample_out, size_t sample) {
    try {
        flat_scene scene = timing_scene(d);
        validate_flat_scene(scene);
        if(!count || reps < 1) throw std::invalid_argument("no rays or no timed launches");
        device_scene uploaded(scene);
        device_buffer<trace_result> output(count);
        const ray *rays = reinterpret_cast<const ray *>(device_rays);
        const unsigned grid = unsigned((count + 255) / 256);
        for(int k = 0; k < warmup; k++) query_rays<<<grid, 256>>>(uploaded.view, rays, output.get(), count, false);
        CUDA_CHECK(cudaGetLastError());
        event start, stop;
        CUDA_CHECK(cudaDeviceSynchronize());
        CUDA_CHECK(cudaEventRecord(start.value));
        for(int k = 0; k < reps; k++) query_rays<<<grid, 256>>>(uploaded.view, rays, output.get(), count, false);
        CUDA_CHECK(cudaEventRecord(stop.value));
        CUDA_CHECK(cudaGetLastError());
        CUDA_CHECK(cudaEventSynchronize(stop.value));
        float ms = 0;
        CUDA_CHECK(cudaEventElapsedTime(&ms, start.value, stop.value));
        *kernel_ms = ms / float(reps);
        if(sample_out && sample) {
            if(sample > count) sample = count;
            CUDA_CHECK(cudaMemcpy(sample_out, output.get(), sample * sizeof(trace_result), cudaMemcpyDeviceToHost));
        }
        return 0;
    } catch(const std::exception &e) { timing_error = e.what(); return 1; }
}

} // extern "C"
