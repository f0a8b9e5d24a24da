/*
 * pt_oracle.h — CPU oracle for the B200 path-tracing core.  TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's hot path (AdmiralHeathCL/cuda-path-tracer):
 * flattened-BVH traversal, triangle/sphere tests, PCG streams, emitter table, light
 * sampling and the MIS bounce loop.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it, and only as the checker; the product never links it.
 *
 * Pinned against the reference itself: tests compare every function here with the
 * reference's own headers compiled into oracle/_ref/ (see oracle/Makefile) and with the
 * golden fixtures under tests/golden/ that those builds produced.
 */
#ifndef PT_ORACLE_H
#define PT_ORACLE_H

#include <stddef.h>
#include <stdint.h>
#include "../include/pt.h"

#ifdef __cplusplus
extern "C" {
#endif

/* scene_view, src/renderer/scene_view.h:31-42 */
typedef struct or_view {
    const pt_triangle *triangles;
    const pt_sphere *spheres;
    const pt_node *nodes;
    const pt_material *materials;
    const pt_texture *textures;
    const unsigned char *pixels;
    int32_t root, node_count;
    const pt_light *lights;
    int32_t light_count;
    float light_area;
} or_view;

typedef struct or_rng { uint64_t state, increment; } or_rng;

/* src/flat/flat_validate.h:10-83: 0 when valid, 1 when the reference would throw. */
int or_validate(const pt_scene_desc *scene);
/* src/renderer/scene_view.h:10-28: returns the number of lights (<= capacity written);
 * *status = 1 when the reference would throw "light area exceeds range". */
size_t or_scene_lights(const pt_scene_desc *scene, pt_light *out, size_t capacity, float *total_area, int *status);

/* src/renderer/random.h */
void or_rng_seed(or_rng *r, uint64_t value, uint64_t pixel);
uint32_t or_rng_next(or_rng *r);
float or_rng_uniform(or_rng *r);

/* src/renderer/transport.h:14-31 */
int or_trace_box(const pt_node *n, const pt_ray *r, float low, float high);
/* src/flat/flat_intersect.h:8-67 */
int or_triangle_hit(const pt_triangle *t, const pt_ray *r, float tmin, float tmax, pt_flat_hit *rec);
int or_sphere_hit(const pt_sphere *s, const pt_ray *r, float tmin, float tmax, pt_flat_hit *rec);

/* src/renderer/transport.h:43-85.  tie_lowest=0 keeps the reference's rule (the later
 * depth-first leaf wins an exact-distance tie); tie_lowest=1 keeps the lowest
 * (primitive_type, primitive_id) instead.  boxes/primitives count like trace_stats. */
int or_trace_world(const or_view *s, const pt_ray *r, float low, float high, pt_flat_hit *hit,
                   int brute, int tie_lowest, int *error, int *boxes, int *primitives);

/* Batch query over `count` rays on `threads` host threads.  mode 0: closest hit with the
 * tie rule above; mode 1: any hit (trace_world's boolean over (tmin, tmax)). */
void or_query(const or_view *s, const pt_ray *rays, size_t count, int mode, float tmin,
              const float *tmax, int brute, int tie_lowest, pt_hit *hits, pt_ray_stats *stats,
              int threads);
/* or_query that also writes, per ray, how many other primitives were hit at exactly the
 * closest distance (0 on a miss): ties[i] > 0 marks a ray whose answer a tie rule decides. */
void or_query_ties(const or_view *s, const pt_ray *rays, size_t count, int mode, float tmin,
                   const float *tmax, int brute, int tie_lowest, pt_hit *hits, pt_ray_stats *stats,
                   int32_t *ties, int threads);
/* cuda_query_rays semantics (src/cuda/cuda_renderer.cu:111-120) on the host. */
void or_query_compat(const or_view *s, const pt_ray *rays, size_t count, int brute,
                     pt_trace_result *out, int threads);

/* trace_pixel_sample / trace_color (src/renderer/transport.h:169-239) with the bounce limit
 * as a parameter (the reference's literal is 50).  Returns the sample's radiance. */
void or_trace_pixel_sample(const or_view *s, const pt_camera *c, int x, int y, int width, int height,
                           or_rng *rng, int brute, int debug, int *error, int direct_light,
                           int max_depth, uint64_t *rays, float out_rgb[3]);

/* portable_renderer::add_samples (tests/support/portable_renderer.h:24-36), sharded over
 * pixels on `threads` host threads.  sums (3 floats/pixel) and rng (2 words/pixel) are
 * read and updated in place; *rays is incremented.  Returns 1 on a stack overflow. */
int or_add_samples(const or_view *s, const pt_camera *c, int width, int height, int samples,
                   int brute, int debug, int direct_light, int max_depth, float *sums,
                   uint64_t *rng, uint64_t *rays, int threads);
/* initialize_pixels (src/cuda/cuda_renderer.cu:64-68). */
void or_reset(int width, int height, uint64_t seed, float *sums, uint64_t *rng);

/* RGBA8 packing.  host_image=0: pack_pixels (src/cuda/cuda_renderer.cu:99-109, sums divided by
 * float(spp)); host_image=1: display_pixels(image()) (src/display/display_pixels.h:11-21 on
 * src/cuda/cuda_renderer.cu:230-234, sums scaled by vec3::operator/= which multiplies by
 * float(1.0/spp)). */
void or_pack_rgba(const float *sums, size_t pixels, int samples, int host_image, unsigned char *rgba);
/* image(): sums scaled by vec3::operator/=(float(spp)) (src/core/vec3.h:152-157). */
void or_image(const float *sums, size_t pixels, int samples, float *rgb);

#ifdef __cplusplus
}
#endif

#endif
