/*
 * pt_oracle.c — CPU oracle (TEST INFRASTRUCTURE ONLY; never linked by the product).
 *
 * Plain-C restatement of the reference's hot path.  Every function cites the reference
 * file:line it follows.  The reference is C++: its float expressions resolve overloads
 * (std::sqrt(float), std::atan2(float,float), …) to float functions, while a few
 * expressions promote to double (M_PI arithmetic, pow(float,int), the 1.0/t inside
 * vec3::operator/=, the 0.001 and 255.0 literals).  This file spells each promotion
 * out, so that compiled without FMA contraction it reproduces the reference's host
 * arithmetic bit for bit.
 */
#define _GNU_SOURCE
#include "pt_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define OR_STACK 64 /* flat_stack_capacity, src/flat/flat_data.h:52 */

/* ------------------------------------------------------------------ vec3 (src/core/vec3.h) */
typedef pt_vec3 v3;
static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mulv(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
/* operator*(float, vec3) and operator*(vec3, float) both compute t*e[i] (vec3.h:126-136) */
static inline v3 muls(float t, v3 v) { return V(t * v.x, t * v.y, t * v.z); }
/* operator/(vec3, float): e[i]/t (vec3.h:130-132) */
static inline v3 divs(v3 v, float t) { return V(v.x / t, v.y / t, v.z / t); }
static inline v3 neg(v3 v) { return V(-v.x, -v.y, -v.z); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) {
    return V(a.y * b.z - a.z * b.y, -(a.x * b.z - a.z * b.x), a.x * b.y - a.y * b.x);
}
static inline float sqlen(v3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
static inline float len(v3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
/* unit_vector(v) = v / v.length() (vec3.h:160-162) */
static inline v3 unit(v3 v) { return divs(v, len(v)); }
/* operator/=(float): k = 1.0/t in double, then e[i] *= float(k) (vec3.h:152-157) */
static inline v3 diveq(v3 v, float t) {
    float k = (float)(1.0 / (double)t);
    return V(v.x * k, v.y * k, v.z * k);
}
static inline float comp(v3 v, int a) { return a == 0 ? v.x : a == 1 ? v.y : v.z; }
static inline int finite3(v3 p) { return isfinite(p.x) && isfinite(p.y) && isfinite(p.z); }
/* ray::point_at_parameter: A + t*B (src/core/ray.h:26-28) */
static inline v3 at(const pt_ray *r, float t) { return add(r->origin, muls(t, r->direction)); }

/* ------------------------------------------------------------------ PCG (src/renderer/random.h:8-23) */
uint32_t or_rng_next(or_rng *r) {
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->increment;
    uint32_t shifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rotation = (uint32_t)(old >> 59u);
    return (shifted >> rotation) | (shifted << ((-rotation) & 31));
}
void or_rng_seed(or_rng *r, uint64_t value, uint64_t pixel) {
    r->state = 0;
    r->increment = (pixel << 1u) | 1u;
    or_rng_next(r);
    r->state += value;
    or_rng_next(r);
}
float or_rng_uniform(or_rng *r) { return (float)(or_rng_next(r) >> 8) * 0x1p-24f; }

/* sample_ball / sample_disk, src/renderer/random.h:25-42 */
static v3 sample_ball(or_rng *r) {
    v3 p;
    do {
        float x = or_rng_uniform(r), y = or_rng_uniform(r), z = or_rng_uniform(r);
        p = sub(muls(2.0f, V(x, y, z)), V(1, 1, 1));
    } while (sqlen(p) >= 1.0f);
    return p;
}
static v3 sample_disk(or_rng *r) {
    v3 p;
    do {
        float x = or_rng_uniform(r), y = or_rng_uniform(r);
        p = sub(muls(2.0f, V(x, y, 0)), V(1, 1, 0));
    } while (sqlen(p) >= 1.0f);
    return p;
}

/* ------------------------------------------------------------------ primitives */
/* get_sphere_uv, src/geometry/sphere_uv.h:7-13 (atan2/asin on float; the rest in double) */
static void sphere_uv(v3 p, float *u, float *v) {
    float phi = atan2f(p.z, p.x);
    float theta = asinf(p.y);
    *u = (float)(1 - ((double)phi + M_PI) / (2 * M_PI));
    *v = (float)(((double)theta + M_PI / 2) / M_PI);
}

/* flat_triangle_hit_geometry, src/flat/flat_intersect.h:8-43 */
int or_triangle_hit(const pt_triangle *face, const pt_ray *r, float t_min, float t_max, pt_flat_hit *rec) {
    v3 edge1 = sub(face->v1, face->v0);
    v3 edge2 = sub(face->v2, face->v0);
    v3 outward = cross(edge1, edge2);
    float normal_length = len(outward);
    float direction_length = len(r->direction);
    if (!(normal_length > 0) || !(direction_length > 0)) return 0;
    v3 pvec = cross(r->direction, edge2);
    float det = dot(edge1, pvec);
    if (fabsf(det) <= 0.0000001f * normal_length * direction_length) return 0;
    float inv_det = 1.0f / det;
    v3 tvec = sub(r->origin, face->v0);
    float u = dot(tvec, pvec) * inv_det;
    if (!(u >= 0 && u <= 1)) return 0;
    v3 qvec = cross(tvec, edge1);
    float v = dot(r->direction, qvec) * inv_det;
    if (!(v >= 0 && u + v <= 1)) return 0;
    float t = dot(edge2, qvec) * inv_det;
    if (!(t > t_min && t < t_max)) return 0;
    outward = diveq(outward, normal_length);
    v3 normal = outward;
    if (face->smooth) {
        float w = 1 - u - v;
        v3 interpolated = add(add(muls(w, face->n0), muls(u, face->n1)), muls(v, face->n2));
        float length_squared = sqlen(interpolated);
        if (length_squared > 0 && isfinite(length_squared)) {
            normal = unit(interpolated);
            if (dot(normal, outward) < 0) normal = neg(normal);
            if (dot(normal, outward) == 0) normal = outward;
        }
    }
    rec->t = t;
    rec->p = at(r, t);
    rec->normal = normal;
    float w = 1 - u - v;
    v3 uv = add(add(muls(w, face->uv0), muls(u, face->uv1)), muls(v, face->uv2));
    rec->u = uv.x;
    rec->v = uv.y;
    rec->material_id = face->material_id;
    return 1;
}

/* flat_sphere_hit, src/flat/flat_intersect.h:49-67 */
int or_sphere_hit(const pt_sphere *s, const pt_ray *r, float t_min, float t_max, pt_flat_hit *rec) {
    v3 oc = sub(r->origin, s->center);
    float a = dot(r->direction, r->direction);
    float b = dot(oc, r->direction);
    float c = dot(oc, oc) - s->radius * s->radius;
    float discriminant = b * b - a * c;
    if (discriminant > 0) {
        float t = (-b - sqrtf(discriminant)) / a;
        if (!(t < t_max && t > t_min)) t = (-b + sqrtf(discriminant)) / a;
        if (t < t_max && t > t_min) {
            rec->t = t;
            rec->p = at(r, t);
            rec->normal = divs(sub(rec->p, s->center), s->radius);
            sphere_uv(rec->normal, &rec->u, &rec->v);
            rec->material_id = s->material_id;
            return 1;
        }
    }
    return 0;
}

/* trace_box, src/renderer/transport.h:14-31 */
int or_trace_box(const pt_node *n, const pt_ray *r, float low, float high) {
    for (int axis = 0; axis < 3; axis++) {
        float d = comp(r->direction, axis);
        float o = comp(r->origin, axis);
        if (d == 0) {
            if (o < comp(n->minimum, axis) || o > comp(n->maximum, axis)) return 0;
            continue;
        }
        float inverse = 1.0f / d;
        float a = (comp(n->minimum, axis) - o) * inverse;
        float b = (comp(n->maximum, axis) - o) * inverse;
        if (inverse < 0) { float swap = a; a = b; b = swap; }
        low = a > low ? a : low;
        high = b < high ? b : high;
        if (high <= low) return 0;
    }
    return high > low;
}

/* trace_leaf, src/renderer/transport.h:33-41 */
static int trace_leaf(const or_view *s, const pt_node *n, const pt_ray *r, float low, float high, pt_flat_hit *hit) {
    int found;
    if (n->type == PT_TRIANGLE) found = or_triangle_hit(&s->triangles[n->primitive], r, low, high, hit);
    else found = or_sphere_hit(&s->spheres[n->primitive], r, low, high, hit);
    if (found) { hit->primitive_type = n->type; hit->primitive_id = n->primitive; }
    return found;
}

static inline int lower_key(const pt_flat_hit *a, const pt_flat_hit *b) {
    if (a->primitive_type != b->primitive_type) return a->primitive_type < b->primitive_type;
    return a->primitive_id < b->primitive_id;
}

/* trace_world, src/renderer/transport.h:43-85.  *ties (may be NULL) receives how many other
 * primitives were hit at exactly the final closest distance: a primitive at that distance is
 * tested whatever the visiting order, because boxes stay eligible up to nextafterf(closest). */
static int trace_world_ties(const or_view *s, const pt_ray *r, float low, float high, pt_flat_hit *hit,
                            int brute, int tie_lowest, int *error, int *boxes, int *primitives, int *ties) {
    int same = 0;
    if (ties) *ties = 0;
    if (s->root < 0) return 0;
    int found = 0;
    float closest = high;
    if (brute) {
        for (int i = 0; i < s->node_count; i++) {
            const pt_node *n = &s->nodes[i];
            if (n->type == PT_BRANCH) continue;
            (*primitives)++;
            pt_flat_hit candidate;
            if (trace_leaf(s, n, r, low, high, &candidate) && (!found || candidate.t <= closest)) {
                same = found && candidate.t == closest ? same + 1 : 0;
                if (tie_lowest && found && candidate.t == closest && !lower_key(&candidate, hit)) continue;
                *hit = candidate; closest = candidate.t; found = 1;
            }
        }
        if (ties) *ties = found ? same : 0;
        return found;
    }
    int stack[OR_STACK], count = 0;
    stack[count++] = s->root;
    while (count) {
        const pt_node *n = &s->nodes[stack[--count]];
        if (n->type == PT_BRANCH) {
            (*boxes)++;
            float limit = found ? nextafterf(closest, high) : high;
            if (!or_trace_box(n, r, low, limit)) continue;
            int needed = n->left == n->right ? 1 : 2;
            if (count + needed > OR_STACK) { *error = 1; return 0; }
            if (n->left != n->right) stack[count++] = n->right;
            stack[count++] = n->left;
        } else {
            (*primitives)++;
            pt_flat_hit candidate;
            float limit = found ? nextafterf(closest, high) : high;
            if (trace_leaf(s, n, r, low, limit, &candidate) && (!found || candidate.t <= closest)) {
                same = found && candidate.t == closest ? same + 1 : 0;
                if (tie_lowest && found && candidate.t == closest && !lower_key(&candidate, hit)) continue;
                *hit = candidate; closest = candidate.t; found = 1;
            }
        }
    }
    if (ties) *ties = found ? same : 0;
    return found;
}

int or_trace_world(const or_view *s, const pt_ray *r, float low, float high, pt_flat_hit *hit,
                   int brute, int tie_lowest, int *error, int *boxes, int *primitives) {
    return trace_world_ties(s, r, low, high, hit, brute, tie_lowest, error, boxes, primitives, NULL);
}

/* ------------------------------------------------------------------ threading helper */
typedef void (*or_range_fn)(void *ctx, size_t begin, size_t end);
typedef struct { or_range_fn fn; void *ctx; size_t begin, end; } or_job;
static void *or_job_main(void *p) { or_job *j = (or_job *)p; j->fn(j->ctx, j->begin, j->end); return NULL; }
static void parallel_for(size_t count, int threads, or_range_fn fn, void *ctx) {
    if (threads < 1) threads = 1;
    if ((size_t)threads > count) threads = count ? (int)count : 1;
    if (threads == 1) { fn(ctx, 0, count); return; }
    pthread_t *ids = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    or_job *jobs = (or_job *)calloc((size_t)threads, sizeof(or_job));
    for (int t = 0; t < threads; t++) {
        jobs[t].fn = fn; jobs[t].ctx = ctx;
        jobs[t].begin = count * (size_t)t / (size_t)threads;
        jobs[t].end = count * (size_t)(t + 1) / (size_t)threads;
        pthread_create(&ids[t], NULL, or_job_main, &jobs[t]);
    }
    for (int t = 0; t < threads; t++) pthread_join(ids[t], NULL);
    free(ids); free(jobs);
}

/* ------------------------------------------------------------------ batch queries */
typedef struct {
    const or_view *s; const pt_ray *rays; int mode; float tmin; const float *tmax;
    int brute, tie_lowest; pt_hit *hits; pt_ray_stats *stats; int32_t *ties;
} query_ctx;
static void query_range(void *p, size_t b, size_t e) {
    query_ctx *q = (query_ctx *)p;
    for (size_t i = b; i < e; i++) {
        pt_flat_hit rec; memset(&rec, 0, sizeof rec);
        int error = 0, boxes = 0, prims = 0, ties = 0;
        float hi = q->tmax ? q->tmax[i] : FLT_MAX;
        int hit = trace_world_ties(q->s, &q->rays[i], q->tmin, hi, &rec, q->brute, q->tie_lowest, &error, &boxes, &prims,
                                   &ties);
        if (q->ties) q->ties[i] = ties;
        pt_hit h;
        h.t = hit ? rec.t : 0.0f;
        h.primitive_id = hit ? rec.primitive_id : -1;
        h.primitive_type = hit ? rec.primitive_type : PT_BRANCH;
        h.error = error;
        if (q->mode == PT_QUERY_ANY) { h.t = 0.0f; h.primitive_id = hit ? 0 : -1; }
        q->hits[i] = h;
        if (q->stats) { q->stats[i].boxes = (uint32_t)boxes; q->stats[i].primitives = (uint32_t)prims; }
    }
}
void or_query_ties(const or_view *s, const pt_ray *rays, size_t count, int mode, float tmin,
                   const float *tmax, int brute, int tie_lowest, pt_hit *hits, pt_ray_stats *stats,
                   int32_t *ties, int threads) {
    query_ctx q = {s, rays, mode, tmin, tmax, brute, tie_lowest, hits, stats, ties};
    parallel_for(count, threads, query_range, &q);
}
void or_query(const or_view *s, const pt_ray *rays, size_t count, int mode, float tmin,
              const float *tmax, int brute, int tie_lowest, pt_hit *hits, pt_ray_stats *stats, int threads) {
    or_query_ties(s, rays, count, mode, tmin, tmax, brute, tie_lowest, hits, stats, NULL, threads);
}

typedef struct { const or_view *s; const pt_ray *rays; int brute; pt_trace_result *out; } compat_ctx;
static void compat_range(void *p, size_t b, size_t e) {
    compat_ctx *q = (compat_ctx *)p;
    for (size_t i = b; i < e; i++) {
        pt_trace_result res;
        memset(&res, 0, sizeof res);
        res.rec.material_id = res.rec.primitive_type = res.rec.primitive_id = -1;
        int error = 0, boxes = 0, prims = 0;
        res.hit = or_trace_world(q->s, &q->rays[i], 0.001f, FLT_MAX, &res.rec, q->brute, 0, &error, &boxes, &prims);
        res.error = error;
        q->out[i] = res;
    }
}
void or_query_compat(const or_view *s, const pt_ray *rays, size_t count, int brute, pt_trace_result *out, int threads) {
    compat_ctx q = {s, rays, brute, out};
    parallel_for(count, threads, compat_range, &q);
}

/* ------------------------------------------------------------------ textures, src/renderer/transport.h:87-111 */
static v3 trace_image(const or_view *scene, const pt_texture *tex, float u, float v) {
    u = fminf(1.0f, fmaxf(0.0f, u));
    v = fminf(1.0f, fmaxf(0.0f, v));
    int i = (int)(u * (float)tex->width);
    int j = (int)((double)((1 - v) * (float)tex->height) - 0.001);
    if (i < 0) i = 0;
    if (j < 0) j = 0;
    if (i > tex->width - 1) i = tex->width - 1;
    if (j > tex->height - 1) j = tex->height - 1;
    size_t offset = (size_t)tex->byte_offset + 3 * (size_t)i + 3 * (size_t)tex->width * (size_t)j;
    float red = (float)((int)scene->pixels[offset] / 255.0);
    float green = (float)((int)scene->pixels[offset + 1] / 255.0);
    float blue = (float)((int)scene->pixels[offset + 2] / 255.0);
    return V(red, green, blue);
}
static v3 trace_texture(const or_view *scene, int32_t id, float u, float v) {
    const pt_texture *tex = &scene->textures[id];
    if (tex->type == PT_TEX_CONSTANT) return tex->color;
    if (tex->type == PT_TEX_IMAGE) return trace_image(scene, tex, u, v);
    u = u * tex->scale.x + tex->offset.x;
    v = v * tex->scale.y + tex->offset.y;
    if (!tex->clamp) { u -= floorf(u); v -= floorf(v); }
    return mulv(tex->color, trace_image(scene, &scene->textures[tex->image_id], u, v));
}

/* ------------------------------------------------------------------ light sampling, src/renderer/light_sampling.h */
static float mis_weight(float a, float b) {
    float scale = fmaxf(a, b);
    if (!(scale > 0)) return 0;
    a /= scale; b /= scale;
    return a * a / (a * a + b * b);
}
static v3 cosine_direction(v3 normal, or_rng *random) {
    float u = or_rng_uniform(random), v = or_rng_uniform(random);
    float radius = sqrtf(u), angle = 2 * (float)M_PI * v;
    v3 helper = fabsf(normal.x) > 0.9f ? V(0, 1, 0) : V(1, 0, 0);
    v3 tangent = unit(cross(helper, normal));
    v3 bitangent = cross(normal, tangent);
    return add(add(muls(radius * cosf(angle), tangent), muls(radius * sinf(angle), bitangent)),
               muls(sqrtf(1 - u), normal));
}
typedef struct { v3 point, normal; float u, v; int material; } light_sample;
static light_sample sample_light(const or_view *scene, or_rng *random) {
    float choice = or_rng_uniform(random) * scene->light_area;
    int low = 0, high = scene->light_count - 1;
    while (low < high) {
        int middle = low + (high - low) / 2;
        if (choice < scene->lights[middle].cumulative_area) high = middle;
        else low = middle + 1;
    }
    const pt_light *light = &scene->lights[low];
    float u = or_rng_uniform(random), v = or_rng_uniform(random);
    light_sample result;
    if (light->type == PT_TRIANGLE) {
        const pt_triangle *t = &scene->triangles[light->primitive];
        float root = sqrtf(u), a = 1 - root, b = root * (1 - v), c = root * v;
        result.point = add(add(muls(a, t->v0), muls(b, t->v1)), muls(c, t->v2));
        result.normal = unit(cross(sub(t->v1, t->v0), sub(t->v2, t->v0)));
        v3 uv = add(add(muls(a, t->uv0), muls(b, t->uv1)), muls(c, t->uv2));
        result.u = uv.x; result.v = uv.y; result.material = t->material_id;
    } else {
        const pt_sphere *s = &scene->spheres[light->primitive];
        float z = 1 - 2 * u, radius = sqrtf(fmaxf(0, 1 - z * z)), angle = 2 * (float)M_PI * v;
        result.normal = V(radius * cosf(angle), z, radius * sinf(angle));
        result.point = add(s->center, muls(fabsf(s->radius), result.normal));
        if (s->radius < 0) result.normal = neg(result.normal);
        sphere_uv(result.normal, &result.u, &result.v);
        result.material = s->material_id;
    }
    return result;
}
static float light_direction_pdf(float area, v3 from, v3 point, v3 normal) {
    v3 delta = sub(point, from);
    float distance_squared = sqlen(delta);
    if (!(area > 0) || !(distance_squared > 0)) return 0;
    float cosine = fabsf(dot(normal, delta)) / sqrtf(distance_squared);
    if (!(cosine > 0)) return 0;
    float pdf = distance_squared / (cosine * area);
    return isfinite(pdf) ? pdf : 0;
}
static float hit_light_pdf(const or_view *scene, v3 from, const pt_flat_hit *hit) {
    v3 normal = hit->normal;
    if (hit->primitive_type == PT_TRIANGLE) {
        const pt_triangle *t = &scene->triangles[hit->primitive_id];
        normal = unit(cross(sub(t->v1, t->v0), sub(t->v2, t->v0)));
    }
    return light_direction_pdf(scene->light_area, from, hit->p, normal);
}

/* ------------------------------------------------------------------ scatter, src/renderer/transport.h:113-155 */
static v3 reflect(v3 v, v3 n) { return sub(v, muls(2 * dot(v, n), n)); }
static int trace_scatter(const or_view *scene, const pt_material *mat, const pt_ray *incoming,
                         const pt_flat_hit *rec, or_rng *random, v3 *attenuation, pt_ray *scattered) {
    if (mat->type == PT_DIFFUSE) {
        v3 target = add(add(rec->p, rec->normal), sample_ball(random));
        scattered->origin = rec->p; scattered->direction = sub(target, rec->p); scattered->time = incoming->time;
        *attenuation = trace_texture(scene, mat->texture_id, rec->u, rec->v);
        return 1;
    }
    if (mat->type == PT_METAL) {
        v3 reflected = reflect(unit(incoming->direction), rec->normal);
        v3 ball = sample_ball(random);
        scattered->origin = rec->p; scattered->direction = add(reflected, muls(mat->fuzz, ball));
        scattered->time = incoming->time;
        *attenuation = mat->albedo;
        return dot(scattered->direction, rec->normal) > 0;
    }
    if (mat->type == PT_GLASS) {
        v3 outward, refracted = V(0, 0, 0);
        v3 reflected = reflect(incoming->direction, rec->normal);
        float ratio, cosine;
        if (dot(incoming->direction, rec->normal) > 0) {
            outward = neg(rec->normal); ratio = mat->ref_idx;
            cosine = mat->ref_idx * dot(incoming->direction, rec->normal) / len(incoming->direction);
        } else {
            outward = rec->normal; ratio = 1.0f / mat->ref_idx;
            cosine = -dot(incoming->direction, rec->normal) / len(incoming->direction);
        }
        v3 uv = unit(incoming->direction);
        float dt = dot(uv, outward);
        float discriminant = 1.0f - ratio * ratio * (1 - dt * dt);
        float probability = 1;
        if (discriminant > 0) {
            refracted = sub(muls(ratio, sub(uv, muls(dt, outward))), muls(sqrtf(discriminant), outward));
            float r0 = (1 - mat->ref_idx) / (1 + mat->ref_idx);
            r0 *= r0;
            /* std::pow(float,int) promotes to double */
            probability = (float)((double)r0 + (double)(1 - r0) * pow((double)(1 - cosine), 5.0));
        }
        scattered->origin = rec->p; scattered->time = incoming->time;
        if (or_rng_uniform(random) < probability) scattered->direction = reflected;
        else scattered->direction = refracted;
        *attenuation = V(1, 1, 1);
        return 1;
    }
    return 0;
}

/* trace_camera, src/renderer/transport.h:157-162 */
static pt_ray trace_camera(const pt_camera *c, float u, float v, or_rng *random) {
    v3 disk = muls(c->lens_radius, sample_disk(random));
    v3 offset = add(muls(disk.x, c->u), muls(disk.y, c->v));
    float time = c->time0 + or_rng_uniform(random) * (c->time1 - c->time0);
    pt_ray r;
    r.origin = add(c->origin, offset);
    r.direction = sub(sub(add(add(c->lower_left_corner, muls(u, c->horizontal)), muls(v, c->vertical)), c->origin), offset);
    r.time = time;
    return r;
}

/* id_color, src/renderer/transport.h:164-167 */
static v3 id_color(int id) {
    uint32_t bits = ((uint32_t)id + 1u) * 2654435761u;
    return V((float)(bits & 255) / 255.0f, (float)((bits >> 8) & 255) / 255.0f, (float)((bits >> 16) & 255) / 255.0f);
}

/* trace_color, src/renderer/transport.h:169-230 (bounce limit `max_depth`, reference 50) */
static v3 trace_color(pt_ray current, const or_view *scene, or_rng *random, int brute, int debug,
                      int *error, int direct_light, int max_depth, uint64_t *rays) {
    v3 throughput = V(1, 1, 1);
    v3 radiance = V(0, 0, 0);
    float previous_pdf = 0;
    for (int depth = 0; depth <= max_depth; depth++) {
        pt_flat_hit rec;
        memset(&rec, 0, sizeof rec);
        int boxes = 0, prims = 0;
        if (rays) ++*rays;
        int hit = or_trace_world(scene, &current, 0.001f, FLT_MAX, &rec, brute, 0, error, &boxes, &prims);
        if (debug == PT_DEBUG_BVH || debug == PT_DEBUG_INTERSECTIONS) {
            float cost = log2f(1.0f + (float)(debug == PT_DEBUG_BVH ? boxes : prims)) / 10.0f;
            cost = fminf(1, cost);
            return V(cost, cost * cost, 1 - cost);
        }
        if (!hit || *error) return radiance;
        if (debug == PT_DEBUG_NORMALS) return muls(0.5f, add(rec.normal, V(1, 1, 1)));
        if (debug == PT_DEBUG_TRIANGLE) return rec.primitive_type == PT_TRIANGLE ? id_color(rec.primitive_id) : V(0.3f, 0.3f, 0.3f);
        if (debug == PT_DEBUG_MATERIAL) return id_color(rec.material_id);
        const pt_material *mat = &scene->materials[rec.material_id];
        if (mat->type == PT_LIGHT) {
            float weight = previous_pdf > 0 ? mis_weight(previous_pdf, hit_light_pdf(scene, current.origin, &rec)) : 1;
            return add(radiance, mulv(muls(weight, throughput), trace_texture(scene, mat->texture_id, rec.u, rec.v)));
        }
        if (depth == max_depth) break;
        pt_ray scattered;
        v3 attenuation;
        if (direct_light && mat->type == PT_DIFFUSE) {
            attenuation = trace_texture(scene, mat->texture_id, rec.u, rec.v);
            if (scene->light_count) {
                light_sample light = sample_light(scene, random);
                v3 delta = sub(light.point, rec.p);
                float distance = len(delta);
                if (distance > 0.002f && isfinite(distance)) {
                    v3 direction = divs(delta, distance);
                    float cosine = fmaxf(0, dot(rec.normal, direction));
                    float pdf = light_direction_pdf(scene->light_area, rec.p, light.point, light.normal);
                    if (cosine > 0 && pdf > 0) {
                        pt_flat_hit blocker;
                        int sb = 0, sp = 0;
                        if (rays) ++*rays;
                        pt_ray shadow = {rec.p, direction, current.time};
                        int blocked = or_trace_world(scene, &shadow, 0.001f, distance - 0.001f, &blocker, brute, 0, error, &sb, &sp);
                        if (!blocked && !*error) {
                            const pt_material *emitter = &scene->materials[light.material];
                            v3 emission = trace_texture(scene, emitter->texture_id, light.u, light.v);
                            float bsdf_pdf = cosine / (float)M_PI;
                            float scale = bsdf_pdf * mis_weight(pdf, bsdf_pdf) / pdf;
                            radiance = add(radiance, muls(scale, mulv(mulv(throughput, attenuation), emission)));
                        }
                    }
                }
            }
            v3 direction = cosine_direction(rec.normal, random);
            previous_pdf = fmaxf(0, dot(rec.normal, direction)) / (float)M_PI;
            throughput = mulv(throughput, attenuation);
            current.origin = rec.p; current.direction = direction;
            continue;
        }
        previous_pdf = 0;
        if (!trace_scatter(scene, mat, &current, &rec, random, &attenuation, &scattered)) break;
        throughput = mulv(throughput, attenuation);
        current = scattered;
    }
    return radiance;
}

/* trace_pixel_sample, src/renderer/transport.h:232-239 */
void or_trace_pixel_sample(const or_view *s, const pt_camera *c, int x, int y, int width, int height,
                           or_rng *rng, int brute, int debug, int *error, int direct_light,
                           int max_depth, uint64_t *rays, float out_rgb[3]) {
    float u = ((float)x + or_rng_uniform(rng)) / (float)width;
    float v = ((float)y + or_rng_uniform(rng)) / (float)height;
    pt_ray r = trace_camera(c, u, v, rng);
    v3 color = trace_color(r, s, rng, brute, debug, error, direct_light, max_depth, rays);
    out_rgb[0] = color.x; out_rgb[1] = color.y; out_rgb[2] = color.z;
}

/* ------------------------------------------------------------------ progressive renderer */
typedef struct {
    const or_view *s; const pt_camera *c; int width, height, samples, brute, debug, direct_light, max_depth;
    float *sums; uint64_t *rng; uint64_t rays[256]; int errors[256]; size_t chunk;
} render_ctx;
static void render_range(void *p, size_t b, size_t e) {
    render_ctx *q = (render_ctx *)p;
    size_t slot = q->chunk ? b / q->chunk : 0;
    if (slot > 255) slot = 255;
    uint64_t rays = 0;
    int failed = 0;
    for (size_t i = b; i < e; i++) {
        int x = (int)(i % (size_t)q->width), y = (int)(i / (size_t)q->width);
        or_rng rng = {q->rng[2 * i], q->rng[2 * i + 1]};
        float acc[3] = {q->sums[3 * i], q->sums[3 * i + 1], q->sums[3 * i + 2]};
        int error = 0;
        for (int s = 0; s < q->samples; s++) {
            float c[3];
            or_trace_pixel_sample(q->s, q->c, x, y, q->width, q->height, &rng, q->brute, q->debug, &error,
                                  q->direct_light, q->max_depth, &rays, c);
            acc[0] += c[0]; acc[1] += c[1]; acc[2] += c[2];
        }
        if (error) failed = 1;
        q->sums[3 * i] = acc[0]; q->sums[3 * i + 1] = acc[1]; q->sums[3 * i + 2] = acc[2];
        q->rng[2 * i] = rng.state; q->rng[2 * i + 1] = rng.increment;
    }
    __atomic_fetch_add(&q->rays[slot], rays, __ATOMIC_RELAXED);
    if (failed) q->errors[slot] = 1;
}
int or_add_samples(const or_view *s, const pt_camera *c, int width, int height, int samples,
                   int brute, int debug, int direct_light, int max_depth, float *sums,
                   uint64_t *rng, uint64_t *rays, int threads) {
    render_ctx *q = (render_ctx *)calloc(1, sizeof(render_ctx));
    size_t count = (size_t)width * (size_t)height;
    q->s = s; q->c = c; q->width = width; q->height = height; q->samples = samples; q->brute = brute;
    q->debug = debug; q->direct_light = direct_light; q->max_depth = max_depth; q->sums = sums; q->rng = rng;
    if (threads > 256) threads = 256;
    if (threads < 1) threads = 1;
    q->chunk = (count + (size_t)threads - 1) / (size_t)threads;
    /* shard in interleaved blocks of rows for balance, one range per thread */
    parallel_for(count, threads, render_range, q);
    uint64_t total = 0;
    int failed = 0;
    for (int i = 0; i < 256; i++) { total += q->rays[i]; failed |= q->errors[i]; }
    *rays += total;
    free(q);
    return failed;
}

void or_reset(int width, int height, uint64_t seed, float *sums, uint64_t *rng) {
    size_t count = (size_t)width * (size_t)height;
    for (size_t i = 0; i < count; i++) {
        or_rng r;
        or_rng_seed(&r, seed, (uint64_t)i);
        sums[3 * i] = sums[3 * i + 1] = sums[3 * i + 2] = 0;
        rng[2 * i] = r.state; rng[2 * i + 1] = r.increment;
    }
}

/* color_channel, src/display/color.h:6-11 */
static int color_channel(float linear) {
    if (!(linear > 0)) return 0;
    if (linear >= 1) return 255;
    float gamma_corrected = sqrtf(linear);
    return (int)(255.99 * (double)gamma_corrected);
}
void or_image(const float *sums, size_t pixels, int samples, float *rgb) {
    for (size_t i = 0; i < pixels; i++) {
        v3 v = V(sums[3 * i], sums[3 * i + 1], sums[3 * i + 2]);
        if (samples) v = diveq(v, (float)samples);
        rgb[3 * i] = v.x; rgb[3 * i + 1] = v.y; rgb[3 * i + 2] = v.z;
    }
}
void or_pack_rgba(const float *sums, size_t pixels, int samples, int host_image, unsigned char *rgba) {
    for (size_t i = 0; i < pixels; i++) {
        v3 v = V(sums[3 * i], sums[3 * i + 1], sums[3 * i + 2]);
        if (host_image) {
            if (samples) v = diveq(v, (float)samples);
            rgba[4 * i] = (unsigned char)color_channel(v.x);
            rgba[4 * i + 1] = (unsigned char)color_channel(v.y);
            rgba[4 * i + 2] = (unsigned char)color_channel(v.z);
        } else {
            /* pack_pixels, src/cuda/cuda_renderer.cu:99-109 */
            v3 color = samples ? divs(v, (float)samples) : V(0, 0, 0);
            for (int ch = 0; ch < 3; ch++) {
                float value = comp(color, ch);
                float gamma = value > 0 && value < 1 ? sqrtf(value) : 0;
                rgba[4 * i + ch] = (unsigned char)(!(value > 0) ? 0 : value >= 1 ? 255 : (int)(255.99 * (double)gamma));
            }
        }
        rgba[4 * i + 3] = 255;
    }
}

/* ------------------------------------------------------------------ scene tables */
/* scene_lights, src/renderer/scene_view.h:10-28 */
size_t or_scene_lights(const pt_scene_desc *s, pt_light *out, size_t capacity, float *total_area, int *status) {
    double area = 0;
    size_t n = 0;
    *status = 0;
    for (size_t i = 0; i < s->triangle_count; i++) {
        const pt_triangle *t = &s->triangles[i];
        if (s->materials[t->material_id].type != PT_LIGHT) continue;
        double size = 0.5 * (double)len(cross(sub(t->v1, t->v0), sub(t->v2, t->v0)));
        if (!(size > 0) || !isfinite(size)) continue;
        area += size;
        if (!isfinite(area) || area > FLT_MAX) { *status = 1; return n; }
        if (n < capacity) { out[n].type = PT_TRIANGLE; out[n].primitive = (int32_t)i; out[n].cumulative_area = (float)area; }
        n++;
    }
    for (size_t i = 0; i < s->sphere_count; i++) {
        const pt_sphere *p = &s->spheres[i];
        if (s->materials[p->material_id].type != PT_LIGHT) continue;
        double size = 4 * M_PI * (double)p->radius * p->radius;
        if (!(size > 0) || !isfinite(size)) continue;
        area += size;
        if (!isfinite(area) || area > FLT_MAX) { *status = 1; return n; }
        if (n < capacity) { out[n].type = PT_SPHERE; out[n].primitive = (int32_t)i; out[n].cumulative_area = (float)area; }
        n++;
    }
    *total_area = n ? (float)area : 0.0f;
    if (n && n <= capacity) *total_area = out[n - 1].cumulative_area;
    return n;
}

/* validate_flat_scene, src/flat/flat_validate.h:10-83 */
typedef struct { const pt_scene_desc *s; int *heights; unsigned char *active; size_t visited; int bad; } val_ctx;
static int valid_id(int32_t id, size_t count) { return id >= 0 && (size_t)id < count; }
static int visit(val_ctx *c, int32_t id, int depth) {
    const pt_scene_desc *s = c->s;
    if (c->bad) return 0;
    if (!(valid_id(id, s->node_count) && depth <= OR_STACK && !c->active[id])) { c->bad = 1; return 0; }
    if (c->heights[id]) {
        if (!(depth + c->heights[id] - 1 <= OR_STACK)) c->bad = 1;
        return c->heights[id];
    }
    c->active[id] = 1;
    c->visited++;
    const pt_node *n = &s->nodes[id];
    if (!(finite3(n->minimum) && finite3(n->maximum))) { c->bad = 1; return 0; }
    for (int a = 0; a < 3; a++) if (!(comp(n->minimum, a) <= comp(n->maximum, a))) { c->bad = 1; return 0; }
    int height = 1;
    if (n->type == PT_BRANCH) {
        int left = visit(c, n->left, depth + 1);
        if (c->bad) return 0;
        int right = n->left == n->right ? left : visit(c, n->right, depth + 1);
        if (c->bad) return 0;
        height += left > right ? left : right;
        int32_t kids[2] = {n->left, n->right};
        for (int k = 0; k < 2; k++) {
            const pt_node *ch = &s->nodes[kids[k]];
            for (int a = 0; a < 3; a++) {
                if (!(comp(n->minimum, a) <= comp(ch->minimum, a) && comp(n->maximum, a) >= comp(ch->maximum, a))) { c->bad = 1; return 0; }
            }
        }
    } else if (n->type == PT_TRIANGLE) {
        if (!valid_id(n->primitive, s->triangle_count)) { c->bad = 1; return 0; }
        const pt_triangle *t = &s->triangles[n->primitive];
        v3 ps[3] = {t->v0, t->v1, t->v2};
        for (int k = 0; k < 3; k++)
            for (int a = 0; a < 3; a++)
                if (!(comp(ps[k], a) >= comp(n->minimum, a) && comp(ps[k], a) <= comp(n->maximum, a))) { c->bad = 1; return 0; }
    } else if (n->type == PT_SPHERE) {
        if (!valid_id(n->primitive, s->sphere_count)) { c->bad = 1; return 0; }
        const pt_sphere *sp = &s->spheres[n->primitive];
        for (int a = 0; a < 3; a++)
            if (!(comp(sp->center, a) - sp->radius >= comp(n->minimum, a) && comp(sp->center, a) + sp->radius <= comp(n->maximum, a))) { c->bad = 1; return 0; }
    } else { c->bad = 1; return 0; }
    c->active[id] = 0;
    c->heights[id] = height;
    return height;
}
int or_validate(const pt_scene_desc *s) {
    for (size_t i = 0; i < s->texture_count; i++) {
        const pt_texture *t = &s->textures[i];
        if (!(finite3(t->color) && finite3(t->scale) && finite3(t->offset))) return 1;
        if (!(t->type >= PT_TEX_CONSTANT && t->type <= PT_TEX_MAP)) return 1;
        if (t->type == PT_TEX_IMAGE) {
            if (!(t->width > 0 && t->height > 0 && t->byte_offset >= 0)) return 1;
            uint64_t end = (uint64_t)t->byte_offset + 3 * (uint64_t)t->width * (uint64_t)t->height;
            if (!(end <= s->pixel_bytes)) return 1;
        } else if (t->type == PT_TEX_MAP) {
            if (!valid_id(t->image_id, s->texture_count)) return 1;
            if (!(s->textures[t->image_id].type == PT_TEX_IMAGE && (t->clamp == 0 || t->clamp == 1))) return 1;
        }
    }
    for (size_t i = 0; i < s->material_count; i++) {
        const pt_material *m = &s->materials[i];
        if (!(m->type >= PT_DIFFUSE && m->type <= PT_LIGHT && finite3(m->albedo))) return 1;
        if (!(isfinite(m->fuzz) && isfinite(m->ref_idx))) return 1;
        if ((m->type == PT_DIFFUSE || m->type == PT_LIGHT) && !valid_id(m->texture_id, s->texture_count)) return 1;
        if (m->type == PT_GLASS && !(m->ref_idx > 0)) return 1;
    }
    for (size_t i = 0; i < s->triangle_count; i++) {
        const pt_triangle *t = &s->triangles[i];
        if (!(valid_id(t->material_id, s->material_count) && (t->smooth == 0 || t->smooth == 1))) return 1;
        if (!(finite3(t->v0) && finite3(t->v1) && finite3(t->v2) && finite3(t->n0) && finite3(t->n1) && finite3(t->n2))) return 1;
        if (!(finite3(t->uv0) && finite3(t->uv1) && finite3(t->uv2))) return 1;
    }
    for (size_t i = 0; i < s->sphere_count; i++) {
        const pt_sphere *p = &s->spheres[i];
        if (!(valid_id(p->material_id, s->material_count) && finite3(p->center) && isfinite(p->radius) && p->radius > 0)) return 1;
    }
    if (s->root == -1) {
        return (s->node_count == 0 && s->triangle_count == 0 && s->sphere_count == 0 && s->max_depth == 0) ? 0 : 1;
    }
    if (!valid_id(s->root, s->node_count)) return 1;
    val_ctx c;
    c.s = s; c.visited = 0; c.bad = 0;
    c.heights = (int *)calloc(s->node_count, sizeof(int));
    c.active = (unsigned char *)calloc(s->node_count, 1);
    int depth = visit(&c, s->root, 1);
    int bad = c.bad || !(depth == s->max_depth && c.visited == s->node_count);
    free(c.heights); free(c.active);
    return bad ? 1 : 0;
}
