/*
 * pt_workloads.h — host-side scene tools of the B200 path-tracing core.
 *
 * The reference builds scenes from OBJ/MTL through its own pointer BVH and flattens them
 * (src/bvh/bvh.h:132-171, src/flat/flat_export.h:13-124); these entry points produce the same
 * flat format for the benchmark workloads, with a binned-SAH tree in place of the random
 * median split.  They need no GPU.  Ray generators that must agree bit-for-bit between host
 * and device use only +, -, *, / and sqrt (no transcendental functions).
 */
#ifndef PT_B200_WORKLOADS_H
#define PT_B200_WORKLOADS_H

#include "pt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pt_flat pt_flat; /* host-owned flat scene (the reference's flat_scene) */

/* Copies the arrays of `desc`; nodes/root/max_depth are kept as given. */
pt_status pt_flat_from_desc(const pt_scene_desc *desc, pt_flat **out);
/* Replaces the node array with a binned-SAH tree over all triangles and spheres
 * (one primitive per leaf, preorder, padded triangle bounds, depth <= 64). threads <= 0: all. */
pt_status pt_flat_build_bvh(pt_flat *scene, int threads);
/* The same output as pt_flat_build_bvh, built mostly on the GPU: 63-bit Morton codes of the
 * primitive box centroids and a radix sort, then rounds of locally-ordered agglomerative
 * clustering (each cluster merges with its mutual nearest neighbour by merged surface area among
 * the 16 clusters on either side in Morton order) until a quarter of the primitives' count remains,
 * then the binned-SAH split of those cluster boxes on the host; node boxes are unions of the
 * children's.  Much faster to build for large scenes; the tree traverses a few percent slower
 * than the full SAH one.  Needs a CUDA device; fails with PT_INVALID_ARGUMENT if the tree would be
 * deeper than 64 levels. */
pt_status pt_flat_build_bvh_gpu(pt_flat *scene);
/* Pointers into the scene's arrays (valid until pt_flat_destroy). */
pt_status pt_flat_desc(const pt_flat *scene, pt_scene_desc *desc);
pt_status pt_flat_destroy(pt_flat *scene);

/* Reference thin-lens camera (src/core/camera.h:16-43), flattened (flatten_camera). */
pt_status pt_make_camera(const float lookfrom[3], const float lookat[3], const float vup[3], float vfov_degrees,
                         float aspect, float aperture, float focus_dist, float time0, float time1, pt_camera *out);

/* Cornell-style box: 10 axis-aligned quads (20 triangles) — floor, back, front, red left,
 * green right walls, a ceiling of 4 quads around a 0.13 x 0.11 emissive quad of radiance 15 —
 * plus a diffuse (r = 0.18), a metal (fuzz 0.1) and a dielectric (IOR 1.5) sphere. */
pt_status pt_workload_cornell(int width, int height, pt_flat **out, pt_camera *camera);

/* Displaced spheres of 2*segments*(rings-1) triangles each (65,536 at 256 x 129) scattered in a
 * box, with materials drawn per sphere, an optional floor and one emissive quad sized to
 * `light_fraction` of the total area.  The procedural 1M-triangle scene is
 * {16, 256, 129, 10, 0.05, 1, 0.005, seed 1}. */
typedef struct pt_procedural_params {
    int sphere_count, segments, rings;
    float box_size;          /* spheres are centered uniformly in [0, box)^3 */
    float displacement;      /* value-noise amplitude, fraction of the radius */
    float radius_min, radius_max;
    int floor;               /* 2-triangle floor below the box */
    float light_fraction;    /* emissive quad area / total scene area */
    float light_radiance;
    float metal_fraction, glass_fraction;
    uint64_t seed;
    int random_triangles;    /* extra uniformly placed small triangles (soup) */
    float soup_edge_min, soup_edge_max;
    int gpu_bvh;             /* 0: binned-SAH tree built on the host; 1: linear BVH built on the GPU */
} pt_procedural_params;
void pt_procedural_defaults(pt_procedural_params *params);
pt_status pt_workload_procedural(const pt_procedural_params *params, int width, int height,
                                 pt_flat **out, pt_camera *camera);

/* The reference's OBJ import and preview stage (src/scene/obj_loader.h:116-237,
 * src/scene/obj_scene.h:10-31; what `ray_tracer --obj FILE` renders): the OBJ's triangles with
 * its MTL materials (Lambertian with Kd or a Kd-tinted PNG/PPM map_Kd, mirror for illum 3/5/8,
 * glass for illum 4/6/7/9, emitter when Ke > 0), transformed by scale, then X/Y/Z rotation in
 * degrees, then translation (any of the three may be NULL), a ground sphere (albedo 0.55) and an
 * emitting sphere (radiance 3) sized to the mesh, and the 40-degree camera that frames it for a
 * width x height image.  Binned-SAH BVH.  Warnings (simplified materials, skipped faces) go to
 * `warnings` (may be NULL).  JPEG textures are rejected (PT_INVALID_ARGUMENT). */
pt_status pt_workload_obj(const char *path, int width, int height, const float scale[3], const float rotate[3],
                          const float translate[3], pt_flat **out, pt_camera *camera, char *warnings, size_t capacity);

/* Camera rays of an image, one PCG stream per ray: ray k covers pixel k mod (w*h), jittered like
 * trace_pixel_sample (src/renderer/transport.h:232-239) with its stream seeded (seed, first+k). */
pt_status pt_rays_camera(const pt_camera *camera, int width, int height, uint64_t seed, uint64_t first,
                         size_t count, pt_ray *rays);
/* Rays leaving random surface points (triangle uniform by index, point uniform by area) with
 * cosine-distributed directions about a randomly oriented geometric normal.  With shadow_tmax
 * non-NULL the rays instead aim at a second surface point and shadow_tmax[k] = distance - 0.001,
 * like the shadow query of src/renderer/transport.h:206-208. */
pt_status pt_rays_surface(const pt_flat *scene, uint64_t seed, uint64_t first, size_t count,
                          pt_ray *rays, float *shadow_tmax, int threads);

/* pt_rays_camera for arbitrary ray indices: rays[k] is the camera ray with index[k] (a random
 * sample of a larger ray set, for bounded CPU checks and baselines). */
pt_status pt_rays_camera_at(const pt_camera *camera, int width, int height, uint64_t seed, const uint64_t *index,
                            size_t count, pt_ray *rays);

/* Bounce rays from closest hits (host form of pt_rays_bounce_device, bit-identical): origin at
 * the hit, a cosine-distributed direction about the geometric normal turned toward the ray, PCG
 * stream (seed, first + k); a miss becomes a random surface ray. */
pt_status pt_rays_bounce(const pt_flat *scene, const pt_ray *primary, const pt_hit *hits, size_t count,
                         uint64_t seed, uint64_t first, pt_ray *rays, int threads);
/* pt_rays_bounce with an explicit PCG stream index per ray (streams[k] in place of first + k). */
pt_status pt_rays_bounce_at(const pt_flat *scene, const pt_ray *primary, const pt_hit *hits, size_t count,
                            uint64_t seed, const uint64_t *streams, pt_ray *rays, int threads);

#ifdef __cplusplus
}
#endif

#endif
