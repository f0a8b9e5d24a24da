// pt_exact.h — FP32 vector arithmetic with the reference's exact operation order.
//
// The reference evaluates its vec3 operators (src/core/vec3.h:101-164) left to right, with
// no fused multiply-add (its CUDA file is built with --fmad=false, CMakeLists.txt:19-20; its
// host code targets baseline x86-64, which has no FMA).  Every translation unit of this
// library that includes this header is compiled with --fmad=false (nvcc) or
// -ffp-contract=off (g++), so the expressions below round exactly like the reference's.
#pragma once

#include <cmath>
#include <cstdint>
#include "pt_internal.h"

namespace ptb {

struct f3 { float x, y, z; };

PT_HD inline f3 mk(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
PT_HD inline f3 mk(const pt_vec3 &v) { return mk(v.x, v.y, v.z); }
PT_HD inline pt_vec3 pv(f3 v) { pt_vec3 r; r.x = v.x; r.y = v.y; r.z = v.z; return r; }
PT_HD inline f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
PT_HD inline f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
PT_HD inline f3 operator-(f3 a) { return mk(-a.x, -a.y, -a.z); }
PT_HD inline f3 operator*(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
// float*vec3 and vec3*float both compute t*e[i]
PT_HD inline f3 operator*(float t, f3 v) { return mk(t * v.x, t * v.y, t * v.z); }
PT_HD inline f3 operator*(f3 v, float t) { return mk(t * v.x, t * v.y, t * v.z); }
// vec3/float divides each component (vec3.h:130-132)
PT_HD inline f3 operator/(f3 v, float t) { return mk(v.x / t, v.y / t, v.z / t); }
PT_HD inline float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PT_HD inline f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - a.z * b.y, -(a.x * b.z - a.z * b.x), a.x * b.y - a.y * b.x);
}
PT_HD inline float sqlen(f3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
PT_HD inline float length(f3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
PT_HD inline f3 unit(f3 v) { return v / length(v); }
// vec3::operator/=(float): multiplies by float(1.0/t), the reciprocal taken in double
PT_HD inline f3 div_assign(f3 v, float t) {
    float k = (float)(1.0 / (double)t);
    return mk(v.x * k, v.y * k, v.z * k);
}
PT_HD inline float comp(f3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
// std::isfinite for float: false for +-inf and NaN
PT_HD inline bool finite(float x) { return fabsf(x) <= 3.402823466e+38f; }

// ---- PCG-XSH-RR 64/32 per pixel stream (src/renderer/random.h:8-23) ----
struct Pcg {
    uint64_t state, increment;
    PT_HD uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + increment;
        uint32_t shifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rotation = (uint32_t)(old >> 59u);
        return (shifted >> rotation) | (shifted << ((-rotation) & 31));
    }
    PT_HD void seed(uint64_t value, uint64_t pixel) {
        state = 0; increment = (pixel << 1u) | 1u;
        next(); state += value; next();
    }
    PT_HD float uniform() { return (float)(next() >> 8) * 0x1p-24f; }
};

// sample_ball / sample_disk rejection samplers (src/renderer/random.h:25-42)
PT_HD inline f3 sample_ball(Pcg &r) {
    f3 p;
    do {
        float x = r.uniform(), y = r.uniform(), z = r.uniform();
        p = 2.0f * mk(x, y, z) - mk(1, 1, 1);
    } while (sqlen(p) >= 1.0f);
    return p;
}
PT_HD inline f3 sample_disk(Pcg &r) {
    f3 p;
    do {
        float x = r.uniform(), y = r.uniform();
        p = 2.0f * mk(x, y, 0) - mk(1, 1, 0);
    } while (sqlen(p) >= 1.0f);
    return p;
}

// trace_camera (src/renderer/transport.h:157-162)
PT_HD inline void camera_ray(const pt_camera &c, float u, float v, Pcg &random, pt_ray &out) {
    f3 disk = c.lens_radius * sample_disk(random);
    f3 offset = mk(c.u) * disk.x + mk(c.v) * disk.y;
    float time = c.time0 + random.uniform() * (c.time1 - c.time0);
    f3 origin = mk(c.origin);
    out.origin = pv(origin + offset);
    out.direction = pv(mk(c.lower_left_corner) + u * mk(c.horizontal) + v * mk(c.vertical) - origin - offset);
    out.time = time;
}

// ---- Per-ray precomputation for the box test. ----
struct RayBox {
    float ox, oy, oz;      // origin
    float ix, iy, iz;      // 1.0f/d per axis, as trace_box computes it (inf for d == 0)
    bool nx, ny, nz;       // inverse < 0: the box's max plane is entered first
};
PT_HD inline RayBox ray_box(const pt_ray &r) {
    RayBox b;
    b.ox = r.origin.x; b.oy = r.origin.y; b.oz = r.origin.z;
    b.ix = 1.0f / r.direction.x; b.iy = 1.0f / r.direction.y; b.iz = 1.0f / r.direction.z;
    b.nx = b.ix < 0; b.ny = b.iy < 0; b.nz = b.iz < 0;
    return b;
}

// trace_box (src/renderer/transport.h:14-31) on an explicit box.  With inverse = 1/d the
// IEEE products reproduce the reference's explicit d == 0 branch: an origin outside the slab
// gives +/-inf and rejects; inside the slab gives -inf..+inf or NaN, which the fmaxf/fminf
// below ignore exactly like `a > low ? a : low` does.  The subtraction and product are
// separate roundings, as in the reference.
PT_HD inline bool box_hit(const RayBox &r, float lox, float hix, float loy, float hiy, float loz,
                          float hiz, float low, float high, float &entry) {
    float ax = ((r.nx ? hix : lox) - r.ox) * r.ix;
    float bx = ((r.nx ? lox : hix) - r.ox) * r.ix;
    float ay = ((r.ny ? hiy : loy) - r.oy) * r.iy;
    float by = ((r.ny ? loy : hiy) - r.oy) * r.iy;
    float az = ((r.nz ? hiz : loz) - r.oz) * r.iz;
    float bz = ((r.nz ? loz : hiz) - r.oz) * r.iz;
    float lo = fmaxf(fmaxf(fmaxf(low, ax), ay), az);
    float hi = fminf(fminf(fminf(high, bx), by), bz);
    entry = lo;
    return hi > lo;
}

// Moller-Trumbore on a pre-transformed triangle (src/flat/flat_intersect.h:8-26).
// dl = |d| of the ray; tri_ok == false when !(dl > 0) (every triangle then misses).
PT_HD inline bool tri_hit(const TriRecord &t, const pt_ray &r, float dl, float tmin, float tmax,
                          float &tout, float &uout, float &vout) {
    f3 d = mk(r.direction);
    f3 e1 = mk(t.e1x, t.e1y, t.e1z), e2 = mk(t.e2x, t.e2y, t.e2z);
    f3 pvec = cross(d, e2);
    float det = dot(e1, pvec);
    if (!(fabsf(det) > t.eps * dl)) return false;
    float inv_det = 1.0f / det;
    f3 tvec = mk(r.origin) - mk(t.v0x, t.v0y, t.v0z);
    float u = dot(tvec, pvec) * inv_det;
    if (!(u >= 0 && u <= 1)) return false;
    f3 qvec = cross(tvec, e1);
    float v = dot(d, qvec) * inv_det;
    if (!(v >= 0 && u + v <= 1)) return false;
    float tt = dot(e2, qvec) * inv_det;
    if (!(tt > tmin && tt < tmax)) return false;
    tout = tt; uout = u; vout = v;
    return true;
}

// flat_sphere_hit distance (src/flat/flat_intersect.h:49-58)
PT_HD inline bool sphere_hit(const SphereRecord &s, const pt_ray &r, float tmin, float tmax, float &tout) {
    f3 d = mk(r.direction);
    f3 oc = mk(r.origin) - mk(s.cx, s.cy, s.cz);
    float a = dot(d, d);
    float b = dot(oc, d);
    float c = dot(oc, oc) - s.radius * s.radius;
    float discriminant = b * b - a * c;
    if (discriminant > 0) {
        float t = (-b - sqrtf(discriminant)) / a;
        if (!(t < tmax && t > tmin)) t = (-b + sqrtf(discriminant)) / a;
        if (t < tmax && t > tmin) { tout = t; return true; }
    }
    return false;
}

// Cosine-distributed direction about n without transcendental functions: a disk point by
// rejection, lifted to the hemisphere (Malley's method), in the tangent frame that
// cosine_direction builds (src/renderer/light_sampling.h:18-25).  Used by the ray generators,
// which must give bit-identical rays on the host and the device.
PT_HD inline f3 cosine_lift(f3 n, Pcg &r) {
    f3 p = sample_disk(r);
    float z = sqrtf(fmaxf(0.0f, 1.0f - p.x * p.x - p.y * p.y));
    f3 helper = fabsf(n.x) > 0.9f ? mk(0, 1, 0) : mk(1, 0, 0);
    f3 tangent = unit(cross(helper, n));
    f3 bitangent = cross(n, tangent);
    return p.x * tangent + p.y * bitangent + z * n;
}

// A surface point: triangle uniform by index, point uniform by area (sqrt warp), geometric
// normal with a random side.
PT_HD inline void surface_point(const pt_triangle *tris, uint64_t count, Pcg &r, f3 &p, f3 &n) {
    const pt_triangle &t = tris[r.next() % count];
    float u = r.uniform(), w = r.uniform();
    float root = sqrtf(u), a = 1 - root, b = root * (1 - w), c = root * w;
    p = a * mk(t.v0) + b * mk(t.v1) + c * mk(t.v2);
    n = unit(cross(mk(t.v1) - mk(t.v0), mk(t.v2) - mk(t.v0)));
    if (r.uniform() < 0.5f) n = -n;
}

// One surface ray (pt_rays_surface / pt_rays_surface_device): origin a random surface point;
// with `shadow`, aimed at a second surface point with *tmax = distance - 0.001 (the shadow query
// of src/renderer/transport.h:206-208), else a cosine-distributed direction about the normal.
PT_HD inline void surface_ray(const pt_triangle *tris, uint64_t count, uint64_t seed, uint64_t index, bool shadow,
                              pt_ray &out, float *tmax) {
    Pcg r; r.seed(seed, index);
    f3 p, n;
    surface_point(tris, count, r, p, n);
    out.origin = pv(p); out.time = 0;
    if (shadow) {
        f3 q, m;
        surface_point(tris, count, r, q, m);
        f3 d = q - p;
        float dist = length(d);
        out.direction = pv(dist > 0 ? d / dist : n);
        *tmax = dist > 0.002f ? dist - 0.001f : 0.001f;
    } else {
        out.direction = pv(cosine_lift(n, r));
    }
}

// One bounce ray (pt_rays_bounce / pt_rays_bounce_device): shared by host and device.
PT_HD inline void bounce_ray(const pt_triangle *tris, uint64_t tri_count, const pt_sphere *spheres, const pt_ray &r,
                             const pt_hit &h, uint64_t seed, uint64_t index, pt_ray &out) {
    Pcg g; g.seed(seed, index);
    f3 p, n;
    f3 d = mk(r.direction);
    if (h.primitive_type == PT_TRIANGLE) {
        const pt_triangle &t = tris[h.primitive_id];
        p = mk(r.origin) + h.t * d;
        n = unit(cross(mk(t.v1) - mk(t.v0), mk(t.v2) - mk(t.v0)));
        if (dot(n, d) > 0) n = -n;
    } else if (h.primitive_type == PT_SPHERE) {
        const pt_sphere &sp = spheres[h.primitive_id];
        p = mk(r.origin) + h.t * d;
        n = (p - mk(sp.center)) / sp.radius;
        if (dot(n, d) > 0) n = -n;
    } else {
        surface_point(tris, tri_count, g, p, n);
    }
    out.origin = pv(p);
    out.direction = pv(cosine_lift(n, g));
    out.time = r.time;
}

} // namespace ptb
