// pt_traverse.h — closest-hit and any-hit traversal of the re-laid-out BVH (host + device).
//
// Semantics follow trace_world (src/renderer/transport.h:43-85):
//   * boxes are tested over (tmin, limit) with limit = nextafterf(closest, tmax) once a hit
//     exists, so exact-distance ties stay eligible (transport.h:65-67);
//   * primitives are tested over (tmin, limit) with the reference's strict bounds;
//   * overflowing the 64-entry stack sets error = 1 and reports a miss (transport.h:71-72).
// What differs is the order, which cannot change the answer: both children's boxes are read
// from the parent (one 64-byte fetch), the nearer passing child is descended first and the
// other pushed, and leaves are tested as soon as their box passes.  Because every
// candidate's t is computed bit-identically and boxes are conservative, the set of
// primitives at the closest distance is independent of the order; among them the winner is
// picked by a key: the lowest (type, id) (the query API's rule) or, for the compatibility
// entry point, the last depth-first leaf (the reference's rule, transport.h:76-79).
#pragma once

#include <cstring>
#include "pt_exact.h"

namespace ptb {

struct HitInfo {
    float t, u, v;
    int32_t slot;   // -1 on a miss
};

#ifdef __CUDA_ARCH__
#define PT_LDG4(p) __ldg(reinterpret_cast<const float4 *>(p))
#define PT_LDGI4(p) __ldg(reinterpret_cast<const int4 *>(p))
#endif

// Smaller key wins an exact-distance tie.  Slots are numbered in the reference walk's
// first-visit order, so the last leaf it reaches has the largest slot.
PT_HD inline long long tie_key(const DeviceScene &s, int32_t slot, int tie) {
    if (tie == kTieLastLeaf) return -(long long)slot;
    if (slot < s.tri_slots) {
        const TriRecord &t = s.tris[slot];
        return tie == kTieLowestId ? ((1ll << 32) | (uint32_t)t.id) : -(long long)t.node;
    }
    const SphereRecord &p = s.spheres[slot - s.tri_slots];
    return tie == kTieLowestId ? ((2ll << 32) | (uint32_t)p.id) : -(long long)p.node;
}

PT_HD inline void load_tri(const DeviceScene &s, int32_t slot, TriRecord &t) {
#ifdef __CUDA_ARCH__
    const float4 *p = reinterpret_cast<const float4 *>(&s.tris[slot]);
    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    t.v0x = a.x; t.v0y = a.y; t.v0z = a.z; t.eps = a.w;
    t.e1x = b.x; t.e1y = b.y; t.e1z = b.z; t.id = __float_as_int(b.w);
    t.e2x = c.x; t.e2y = c.y; t.e2z = c.z; t.node = __float_as_int(c.w);
#else
    t = s.tris[slot];
#endif
}

PT_HD inline void load_node(const DeviceScene &s, int32_t node, BvhNode &n) {
#ifdef __CUDA_ARCH__
    const float4 *p = reinterpret_cast<const float4 *>(&s.nodes[node]);
    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    int4 d = __ldg(reinterpret_cast<const int4 *>(p + 3));
    n.c0lox = a.x; n.c0hix = a.y; n.c0loy = a.z; n.c0hiy = a.w;
    n.c1lox = b.x; n.c1hix = b.y; n.c1loy = b.z; n.c1hiy = b.w;
    n.c0loz = c.x; n.c0hiz = c.y; n.c1loz = c.z; n.c1hiz = c.w;
    n.child0 = d.x; n.child1 = d.y;
#else
    n = s.nodes[node];
#endif
}

// Tests leaf `slot`; updates the running answer.  Returns true when a hit was accepted.  `any`
// selects any-hit (the first hit is the answer) or closest-hit (ties by key) at run time; the
// template below fixes it at compile time.
PT_HD __forceinline__ bool test_leaf_rt(const DeviceScene &s, int32_t slot, const pt_ray &r, float dl, float tmin,
                                        float tmax, int tie, bool any, bool &found, float &closest, long long &best_key,
                                        HitInfo &hit, uint32_t &prims) {
    float limit = found ? nextafterf(closest, tmax) : tmax;
    float t, u = 0, v = 0;
    bool ok;
    prims++;
    if (slot < s.tri_slots) {
        if (!(dl > 0)) return false;   // !(direction_length > 0), flat_intersect.h:14
        TriRecord tr;
        load_tri(s, slot, tr);
        ok = tri_hit(tr, r, dl, tmin, limit, t, u, v);
    } else {
        SphereRecord sp = s.spheres[slot - s.tri_slots];
        ok = sphere_hit(sp, r, tmin, limit, t);
    }
    if (!ok) return false;
    if (!any && found && !(t < closest)) {
        long long key = tie_key(s, slot, tie);
        if (!(key < best_key)) return false;
        best_key = key;
    } else if (!any) {
        best_key = tie_key(s, slot, tie);
    }
    found = true;
    closest = t;
    hit.t = t; hit.u = u; hit.v = v; hit.slot = slot;
    return true;
}
template <bool kAny>
PT_HD __forceinline__ bool test_leaf(const DeviceScene &s, int32_t slot, const pt_ray &r, float dl, float tmin,
                                     float tmax, int tie, bool &found, float &closest, long long &best_key,
                                     HitInfo &hit, uint32_t &prims) {
    return test_leaf_rt(s, slot, r, dl, tmin, tmax, tie, kAny, found, closest, best_key, hit, prims);
}

// Closest hit (any = false) or any hit (any = true) over (tmin, tmax), from node `root` of the
// two-wide array (several trees may share it).
PT_HD inline bool traverse_rt(const DeviceScene &s, const pt_ray &r, float tmin, float tmax, int tie, bool any,
                              HitInfo &hit, uint32_t &boxes, uint32_t &prims, int &error, int32_t root = 0) {
    hit.slot = -1; hit.t = 0; hit.u = 0; hit.v = 0;
    if (s.empty || s.node_count == 0 || root < 0) return false;
    RayBox rb = ray_box(r);
    float dl = length(mk(r.direction));
    bool found = false;
    float closest = tmax;
    long long best_key = 0;
    int32_t stack[kStackCapacity];
    int sp = 0;
    int32_t node = root;
    for (;;) {
        BvhNode n;
        load_node(s, node, n);
        float limit = found ? nextafterf(closest, tmax) : tmax;
        float e0, e1;
        bool h0 = n.child0 != kEmptyChild &&
                  box_hit(rb, n.c0lox, n.c0hix, n.c0loy, n.c0hiy, n.c0loz, n.c0hiz, tmin, limit, e0);
        bool h1 = n.child1 != kEmptyChild &&
                  box_hit(rb, n.c1lox, n.c1hix, n.c1loy, n.c1hiy, n.c1loz, n.c1hiz, tmin, limit, e1);
        boxes += (n.child0 != kEmptyChild) + (n.child1 != kEmptyChild);
        int32_t first = n.child0, second = n.child1;
        bool hf = h0, hs = h1;
        if (h0 && h1 && e1 < e0) { first = n.child1; second = n.child0; }
        else if (!h0) { first = n.child1; hf = h1; hs = false; }
        // leaves are tested at once, nearer first
        int32_t inner[2];
        int ninner = 0;
        if (hf) {
            if (first < 0) {
                if (test_leaf_rt(s, ~first, r, dl, tmin, tmax, tie, any, found, closest, best_key, hit, prims) && any) return true;
            } else inner[ninner++] = first;
        }
        if (hs) {
            if (second < 0) {
                if (test_leaf_rt(s, ~second, r, dl, tmin, tmax, tie, any, found, closest, best_key, hit, prims) && any) return true;
            } else inner[ninner++] = second;
        }
        if (ninner == 2) {
            if (sp >= kStackCapacity) { error = 1; hit.slot = -1; return false; }
            stack[sp++] = inner[1];
            node = inner[0];
        } else if (ninner == 1) {
            node = inner[0];
        } else {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
    return found;
}
template <bool kAny>
PT_HD inline bool traverse(const DeviceScene &s, const pt_ray &r, float tmin, float tmax, int tie,
                           HitInfo &hit, uint32_t &boxes, uint32_t &prims, int &error) {
    return traverse_rt(s, r, tmin, tmax, tie, kAny, hit, boxes, prims, error, 0);
}

// trace_world in the reference's own visiting order (src/renderer/transport.h:61-84): a
// branch's box is tested when it is popped, its right child pushed below its left, leaves
// tested without a box test.  Same answer as traverse<>; used where the reference's per-ray
// counts matter (the bvh / intersections debug views count boxes and primitives like its
// trace_stats).  Stack entries are (parent node << 1 | side) so the popped child's box is
// read from its parent.
PT_HD inline bool traverse_reference(const DeviceScene &s, const pt_ray &r, float tmin, float tmax, int tie,
                                     HitInfo &hit, uint32_t &boxes, uint32_t &prims, int &error) {
    hit.slot = -1; hit.t = 0; hit.u = 0; hit.v = 0;
    if (s.empty || s.node_count == 0) return false;
    RayBox rb = ray_box(r);
    float dl = length(mk(r.direction));
    bool found = false;
    float closest = tmax;
    long long best_key = 0;
    if (s.root_leaf) {
        BvhNode n;
        load_node(s, 0, n);
        test_leaf<false>(s, ~n.child0, r, dl, tmin, tmax, tie, found, closest, best_key, hit, prims);
        return found;
    }
    // the root branch: its own box first
    {
        boxes++;
        float e;
        if (!box_hit(rb, s.root_lo[0], s.root_hi[0], s.root_lo[1], s.root_hi[1], s.root_lo[2], s.root_hi[2], tmin, tmax, e))
            return false;
    }
    int32_t stack[kStackCapacity];
    int sp = 0;
    // children of the root: push right (if distinct) then left
    {
        BvhNode n;
        load_node(s, 0, n);
        int needed = n.child1 == kEmptyChild ? 1 : 2;
        if (sp + needed > kStackCapacity) { error = 1; hit.slot = -1; return false; }
        if (n.child1 != kEmptyChild) stack[sp++] = (0 << 1) | 1;
        stack[sp++] = (0 << 1) | 0;
    }
    while (sp) {
        int32_t entry = stack[--sp];
        int32_t parent = entry >> 1, side = entry & 1;
        BvhNode p;
        load_node(s, parent, p);
        int32_t child = side ? p.child1 : p.child0;
        if (child >= 0) {
            boxes++;
            float limit = found ? nextafterf(closest, tmax) : tmax;
            float e;
            bool h = side ? box_hit(rb, p.c1lox, p.c1hix, p.c1loy, p.c1hiy, p.c1loz, p.c1hiz, tmin, limit, e)
                          : box_hit(rb, p.c0lox, p.c0hix, p.c0loy, p.c0hiy, p.c0loz, p.c0hiz, tmin, limit, e);
            if (!h) continue;
            BvhNode n;
            load_node(s, child, n);
            int needed = n.child1 == kEmptyChild ? 1 : 2;
            if (sp + needed > kStackCapacity) { error = 1; hit.slot = -1; return false; }
            if (n.child1 != kEmptyChild) stack[sp++] = (child << 1) | 1;
            stack[sp++] = (child << 1) | 0;
        } else {
            test_leaf<false>(s, ~child, r, dl, tmin, tmax, tie, found, closest, best_key, hit, prims);
        }
    }
    return found;
}

// trace_world(…, brute = true) (src/renderer/transport.h:48-60): every leaf, in flat
// node-array order, without pruning.
template <bool kAny>
PT_HD inline bool traverse_brute(const DeviceScene &s, const int32_t *order, int32_t leaves, const pt_ray &r,
                                 float tmin, float tmax, int tie, HitInfo &hit, uint32_t &prims) {
    hit.slot = -1; hit.t = 0; hit.u = 0; hit.v = 0;
    if (s.empty) return false;
    float dl = length(mk(r.direction));
    bool found = false;
    float closest = tmax;
    long long best_key = 0;
    for (int32_t i = 0; i < leaves; i++) {
        if (test_leaf<kAny>(s, order[i], r, dl, tmin, tmax, tie, found, closest, best_key, hit, prims) && kAny)
            return true;
    }
    return found;
}

// ---- full hit record of the winner (src/flat/flat_intersect.h:27-42, 53-64) ----
PT_HD inline void sphere_uv(f3 p, float &u, float &v) {
    // get_sphere_uv, src/geometry/sphere_uv.h:7-13: atan2/asin on float, the rest in double
    const double pi = 3.14159265358979323846;
    float phi = atan2f(p.z, p.x);
    float theta = asinf(p.y);
    u = (float)(1 - ((double)phi + pi) / (2 * pi));
    v = (float)(((double)theta + pi / 2) / pi);
}

PT_HD inline void finalize_hit(const DeviceScene &s, const pt_ray &r, const HitInfo &h, pt_flat_hit &rec) {
    f3 o = mk(r.origin), d = mk(r.direction);
    rec.t = h.t;
    f3 p = o + h.t * d;
    rec.p = pv(p);
    if (h.slot < s.tri_slots) {
        const TriRecord &tr = s.tris[h.slot];
        const pt_triangle &face = s.triangles[tr.id];
        float u = h.u, v = h.v;
        f3 edge1 = mk(face.v1) - mk(face.v0), edge2 = mk(face.v2) - mk(face.v0);
        f3 outward = cross(edge1, edge2);
        float normal_length = length(outward);
        outward = div_assign(outward, normal_length);
        f3 normal = outward;
        if (face.smooth) {
            f3 interpolated = (1 - u - v) * mk(face.n0) + u * mk(face.n1) + v * mk(face.n2);
            float length_squared = sqlen(interpolated);
            if (length_squared > 0 && finite(length_squared)) {
                normal = unit(interpolated);
                if (dot(normal, outward) < 0) normal = -normal;
                if (dot(normal, outward) == 0) normal = outward;
            }
        }
        rec.normal = pv(normal);
        f3 uv = (1 - u - v) * mk(face.uv0) + u * mk(face.uv1) + v * mk(face.uv2);
        rec.u = uv.x; rec.v = uv.y;
        rec.material_id = face.material_id;
        rec.primitive_type = PT_TRIANGLE;
        rec.primitive_id = tr.id;
    } else {
        const SphereRecord &sr = s.spheres[h.slot - s.tri_slots];
        const pt_sphere &sp = s.sphere_src[sr.id];
        f3 normal = (p - mk(sp.center)) / sp.radius;
        rec.normal = pv(normal);
        sphere_uv(normal, rec.u, rec.v);
        rec.material_id = sp.material_id;
        rec.primitive_type = PT_SPHERE;
        rec.primitive_id = sr.id;
    }
}

PT_HD inline void hit_ids(const DeviceScene &s, int32_t slot, int32_t &type, int32_t &id) {
    if (slot < 0) { type = PT_BRANCH; id = -1; return; }
    if (slot < s.tri_slots) { type = PT_TRIANGLE; id = s.tris[slot].id; return; }
    type = PT_SPHERE; id = s.spheres[slot - s.tri_slots].id;
}

} // namespace ptb

namespace ptb {

// Resumable closest-hit / any-hit traversal: the same walk as traverse<>, cut into steps of
// one node each so a persistent warp can retire finished rays and take new ones between
// steps (the lanes of a warp then stay busy until the ray pool is empty).
struct Walker {
    RayBox rb;
    pt_ray r;
    float dl, tmin, tmax, closest;
    long long best_key;
    HitInfo hit;
    uint32_t boxes, prims;
    int32_t node, sp;
    bool found;
    int error;
    int32_t stack[kStackCapacity];

    PT_HD void begin(const DeviceScene &s, const pt_ray &ray, float lo, float hi) {
        r = ray; rb = ray_box(ray); dl = length(mk(ray.direction));
        tmin = lo; tmax = hi; closest = hi; best_key = 0;
        hit.slot = -1; hit.t = 0; hit.u = 0; hit.v = 0;
        boxes = 0; prims = 0; sp = 0; found = false; error = 0;
        node = (s.empty || s.node_count == 0) ? -1 : 0;
    }
    // One node: both child boxes, leaf children tested at once (nearer first), descend into
    // the nearer inner child and push the other.  Returns true when the walk has ended.
    template <bool kAny>
    PT_HD bool step(const DeviceScene &s, int tie) {
        if (node < 0) return true;
        BvhNode n;
        load_node(s, node, n);
        float limit = found ? nextafterf(closest, tmax) : tmax;
        float e0, e1;
        bool h0 = n.child0 != kEmptyChild && box_hit(rb, n.c0lox, n.c0hix, n.c0loy, n.c0hiy, n.c0loz, n.c0hiz, tmin, limit, e0);
        bool h1 = n.child1 != kEmptyChild && box_hit(rb, n.c1lox, n.c1hix, n.c1loy, n.c1hiy, n.c1loz, n.c1hiz, tmin, limit, e1);
        boxes += (n.child0 != kEmptyChild) + (n.child1 != kEmptyChild);
        int32_t first = n.child0, second = n.child1;
        bool hf = h0, hs = h1;
        if (h0 && h1 && e1 < e0) { first = n.child1; second = n.child0; }
        else if (!h0) { first = n.child1; hf = h1; hs = false; }
        int32_t inner[2];
        int ninner = 0;
        if (hf) {
            if (first < 0) {
                if (test_leaf<kAny>(s, ~first, r, dl, tmin, tmax, tie, found, closest, best_key, hit, prims) && kAny) { node = -1; return true; }
            } else inner[ninner++] = first;
        }
        if (hs) {
            if (second < 0) {
                if (test_leaf<kAny>(s, ~second, r, dl, tmin, tmax, tie, found, closest, best_key, hit, prims) && kAny) { node = -1; return true; }
            } else inner[ninner++] = second;
        }
        if (ninner == 2) {
            if (sp >= kStackCapacity) { error = 1; found = false; hit.slot = -1; node = -1; return true; }
            stack[sp++] = inner[1];
            node = inner[0];
        } else if (ninner == 1) {
            node = inner[0];
        } else {
            if (sp == 0) { node = -1; return true; }
            node = stack[--sp];
        }
        return false;
    }
};

} // namespace ptb

#ifdef __CUDACC__
namespace ptb {

// Entries of each lane's traversal stack kept in shared memory (entry-major, so the lanes of a
// warp touch consecutive words); deeper entries go to local memory.  A near-first walk pushes
// at most one entry per level, so a validated tree (depth <= 64) never needs more than 63.
constexpr int kSharedStack = 32;

// Result of a finished walk, handed to the consumer.
struct WalkResult { float t, u, v; int32_t slot; uint32_t boxes, prims; int error; };

// Persistent warp loop over `count` work items.  Lanes take item indices from *next (one
// atomicAdd per warp); between traversal steps a warp hands new items to idle lanes once fewer
// than `min_active` lanes are busy.  get(k, ray, tmin, tmax) loads item k; done(k, result)
// consumes a finished walk.  Every lane of the warp must call this together, and the block
// must provide kSharedStack * blockDim.x int32 words of dynamic shared memory.  With kRoot, get()
// also returns the walk's root node (several trees in one node array; < 0 for an empty tree).
template <bool kAny, bool kRoot = false, class Get, class Done>
__device__ inline void persistent_walk(const DeviceScene &s, size_t count, unsigned long long *next, int min_active,
                                       int tie, Get get, Done done) {
    // Warps past the first `count` lanes have nothing to take: they leave before touching the
    // shared counter (a short queue then costs a few warps, not the whole resident grid).
    const size_t warp_first = (size_t(blockIdx.x) * blockDim.x + (threadIdx.x & ~31u));
    if (warp_first >= count) return;
    extern __shared__ int32_t shared_stack[];
    int32_t *my_stack = shared_stack + threadIdx.x;
    const int stride = blockDim.x;
    int32_t spill[kStackCapacity - kSharedStack];
    const unsigned lane = threadIdx.x & 31;
    // walk state (registers)
    pt_ray r;
    RayBox rb;
    float dl = 0, tmin = 0, tmax = 0, closest = 0;
    long long best_key = 0;
    HitInfo hit;
    uint32_t boxes = 0, prims = 0;
    int32_t node = -1, sp = 0;
    bool found = false;
    int error = 0;
    size_t index = 0;
    bool busy = false, pool_empty = false;
    hit.slot = -1; hit.t = 0; hit.u = 0; hit.v = 0;
    for (;;) {
        unsigned idle = __ballot_sync(0xffffffffu, !busy);
        if (idle && !pool_empty) {
            int leader = __ffs(idle) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(next, (unsigned long long)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(idle) >= count) pool_empty = true;
            if (!busy) {
                size_t mine = base + __popc(idle & ((1u << lane) - 1u));
                if (mine < count) {
                    index = mine;
                    int32_t root = 0;
                    if constexpr (kRoot) get(index, r, tmin, tmax, root);
                    else get(index, r, tmin, tmax);
                    rb = ray_box(r);
                    dl = length(mk(r.direction));
                    closest = tmax; best_key = 0;
                    hit.slot = -1; hit.t = 0; hit.u = 0; hit.v = 0;
                    boxes = 0; prims = 0; sp = 0; found = false; error = 0;
                    node = (s.empty || s.node_count == 0 || root < 0) ? -1 : root;
                    busy = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, busy)) break;
        const int threshold = pool_empty ? 1 : min_active;
        for (;;) {
            if (busy) {
                bool end = false;
                if (node < 0) end = true;
                else {
                    BvhNode n;
                    load_node(s, node, n);
                    float limit = found ? nextafterf(closest, tmax) : tmax;
                    float e0, e1;
                    bool h0 = n.child0 != kEmptyChild && box_hit(rb, n.c0lox, n.c0hix, n.c0loy, n.c0hiy, n.c0loz, n.c0hiz, tmin, limit, e0);
                    bool h1 = n.child1 != kEmptyChild && box_hit(rb, n.c1lox, n.c1hix, n.c1loy, n.c1hiy, n.c1loz, n.c1hiz, tmin, limit, e1);
                    boxes += (n.child0 != kEmptyChild) + (n.child1 != kEmptyChild);
                    int32_t first = n.child0, second = n.child1;
                    bool hf = h0, hs = h1;
                    if (h0 && h1 && e1 < e0) { first = n.child1; second = n.child0; }
                    else if (!h0) { first = n.child1; hf = h1; hs = false; }
                    int32_t inner0 = -1, inner1 = -1;
                    int ninner = 0;
                    if (hf) {
                        if (first < 0) {
                            if (test_leaf<kAny>(s, ~first, r, dl, tmin, tmax, tie, found, closest, best_key, hit, prims) && kAny) end = true;
                        } else { inner0 = first; ninner = 1; }
                    }
                    if (hs && !end) {
                        if (second < 0) {
                            if (test_leaf<kAny>(s, ~second, r, dl, tmin, tmax, tie, found, closest, best_key, hit, prims) && kAny) end = true;
                        } else { if (ninner) inner1 = second; else inner0 = second; ninner++; }
                    }
                    if (!end) {
                        if (ninner == 2) {
                            if (sp >= kStackCapacity) { error = 1; found = false; hit.slot = -1; end = true; }
                            else {
                                if (sp < kSharedStack) my_stack[sp * stride] = inner1;
                                else spill[sp - kSharedStack] = inner1;
                                sp++;
                                node = inner0;
                            }
                        } else if (ninner == 1) {
                            node = inner0;
                        } else if (sp == 0) {
                            end = true;
                        } else {
                            sp--;
                            node = sp < kSharedStack ? my_stack[sp * stride] : spill[sp - kSharedStack];
                        }
                    }
                }
                if (end) {
                    WalkResult res;
                    res.t = hit.t; res.u = hit.u; res.v = hit.v; res.slot = found ? hit.slot : -1;
                    res.boxes = boxes; res.prims = prims; res.error = error;
                    done(index, res);
                    busy = false;
                    node = -1;
                }
            }
            if (__popc(__ballot_sync(0xffffffffu, busy)) < threshold) break;
        }
    }
}

} // namespace ptb
#endif

namespace ptb {

// ---- four-wide traversal -------------------------------------------------------------------
// Same answer as traverse<> (same primitive tests, same limit rule, same tie keys); fewer,
// wider steps.  A step tests the four child boxes of a node, visits the nearest passing child
// next and pushes the others, farthest first, with their entry distance; a popped entry whose
// entry distance is no longer below the current limit is dropped (the box test repeated with the
// new limit).
// The box tests only filter: a primitive the walk never reaches could change the answer only if
// the ray hit it at a point outside a box around it, and every box holds its primitives' boxes,
// which the reference pads by 1e-4 on every axis (src/geometry/triangle.h:96-109).  So the walk
// reads the children's boxes quantised outward to 8 bits per bound (Bvh4QNode, 64 bytes), and
// computes each slab value in two fused multiply-adds, t = q * (2^e / d) + (p - o) / d, whose
// rounding (a few ulps of t and of o/d) stays far inside that margin for scenes of up to a few
// hundred units; a box passes when entry <= exit.  A zero direction component is replaced by
// +-1e-30 in the box test's inverse, so its slab accepts exactly the origins inside it.

// Per-ray constants of the four-wide box test.
struct RayBox4 {
    float jx, jy, jz;      // 1/d per axis (|d| >= 1e-30)
    float kx, ky, kz;      // -o * (1/d)
    bool nx, ny, nz;       // 1/d < 0: the box's max plane is entered first
};
PT_HD inline RayBox4 ray_box4(const pt_ray &r) {
    auto inv = [](float d) { return 1.0f / (fabsf(d) > 1e-30f ? d : (d < 0.0f ? -1e-30f : 1e-30f)); };
    RayBox4 b;
    b.jx = inv(r.direction.x); b.jy = inv(r.direction.y); b.jz = inv(r.direction.z);
    b.kx = -(r.origin.x * b.jx); b.ky = -(r.origin.y * b.jy); b.kz = -(r.origin.z * b.jz);
    b.nx = b.jx < 0; b.ny = b.jy < 0; b.nz = b.jz < 0;
    return b;
}
PT_HD inline float fma_box(float a, float b, float c) {
#ifdef __CUDA_ARCH__
    return __fmaf_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
PT_HD inline float max3(float a, float b, float c) {
#ifdef __CUDA_ARCH__
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
#else
    return fmaxf(fmaxf(a, b), c);
#endif
}
PT_HD inline float min3(float a, float b, float c) {
#ifdef __CUDA_ARCH__
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
#else
    return fminf(fminf(a, b), c);
#endif
}

#ifdef __CUDA_ARCH__
// eight consecutive words of a 32-byte aligned address, one 256-bit load through the read-only path
__device__ __forceinline__ void ldg8(const float *p, float (&v)[8]) {
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
                 : "l"(p));
}
#endif

PT_HD inline void load_node4(const DeviceScene &s, int32_t node, Bvh4QNode &n) {
#ifdef __CUDA_ARCH__
    const float *p = reinterpret_cast<const float *>(&s.nodes4[node]);   // 64-byte records, 256-byte aligned base
    float x[8], y[8];
    ldg8(p, x);
    ldg8(p + 8, y);
    n.px = x[0]; n.py = x[1]; n.pz = x[2]; n.sx = x[3]; n.sy = y[6]; n.sz = y[7];
    n.qlo[0] = __float_as_uint(x[4]); n.qlo[1] = __float_as_uint(x[5]); n.qlo[2] = __float_as_uint(x[6]);
    n.qhi[0] = __float_as_uint(x[7]); n.qhi[1] = __float_as_uint(y[0]); n.qhi[2] = __float_as_uint(y[1]);
    n.child[0] = __float_as_int(y[2]); n.child[1] = __float_as_int(y[3]); n.child[2] = __float_as_int(y[4]); n.child[3] = __float_as_int(y[5]);
#else
    n = s.nodes4[node];
#endif
}

// byte k of w as a float, exactly (one integer-to-float conversion of the byte on the device)
PT_HD inline float qbyte(uint32_t w, int k) {
#ifdef __CUDA_ARCH__
    return __uint2float_rn((w >> (8 * k)) & 0xffu);
#else
    return float((w >> (8 * k)) & 0xffu);
#endif
}

// Tests the children of `node`; returns how many passed, in `ref`/`dist` sorted nearest first.
PT_HD inline int node4_children(const DeviceScene &s, int32_t node, const RayBox4 &rb, float tmin, float limit,
                                int32_t ref[4], float dist[4], uint32_t &boxes) {
    Bvh4QNode n;
    load_node4(s, node, n);
    const float sx = n.sx * rb.jx, sy = n.sy * rb.jy, sz = n.sz * rb.jz;
    const float tx = fma_box(n.px, rb.jx, rb.kx), ty = fma_box(n.py, rb.jy, rb.ky), tz = fma_box(n.pz, rb.jz, rb.kz);
    const uint32_t nxw = rb.nx ? n.qhi[0] : n.qlo[0], fxw = rb.nx ? n.qlo[0] : n.qhi[0];
    const uint32_t nyw = rb.ny ? n.qhi[1] : n.qlo[1], fyw = rb.ny ? n.qlo[1] : n.qhi[1];
    const uint32_t nzw = rb.nz ? n.qhi[2] : n.qlo[2], fzw = rb.nz ? n.qlo[2] : n.qhi[2];
    int hits = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float ax = fma_box(qbyte(nxw, k), sx, tx), bx = fma_box(qbyte(fxw, k), sx, tx);
        const float ay = fma_box(qbyte(nyw, k), sy, ty), by = fma_box(qbyte(fyw, k), sy, ty);
        const float az = fma_box(qbyte(nzw, k), sz, tz), bz = fma_box(qbyte(fzw, k), sz, tz);
        const float entry = fmaxf(max3(ax, ay, az), tmin), exit = fminf(min3(bx, by, bz), limit);
        const bool h = n.child[k] != kEmptyChild && entry <= exit;
        boxes += n.child[k] != kEmptyChild;
        ref[k] = n.child[k];
        dist[k] = h ? entry : INFINITY;
        hits += h;
    }
    // sorting network on (dist, ref), ascending
#define PT_CSWAP(i, j) if (dist[j] < dist[i]) { float td = dist[i]; dist[i] = dist[j]; dist[j] = td; int32_t tr = ref[i]; ref[i] = ref[j]; ref[j] = tr; }
    PT_CSWAP(0, 1) PT_CSWAP(2, 3) PT_CSWAP(0, 2) PT_CSWAP(1, 3) PT_CSWAP(1, 2)
#undef PT_CSWAP
    return hits;
}

// Tests the 1..8 slots of a leaf reference; true when `any` and a hit was found.
PT_HD __forceinline__ bool leaf4_rt(const DeviceScene &s, int32_t ref, const pt_ray &r, float dl, float tmin, float tmax,
                                    int tie, bool any, bool &found, float &closest, long long &best_key, HitInfo &hit,
                                    uint32_t &prims) {
    int32_t v = ~ref;
    int32_t first = v >> 3, count = (v & 7) + 1;
    for (int32_t j = 0; j < count; j++)
        if (test_leaf_rt(s, first + j, r, dl, tmin, tmax, tie, any, found, closest, best_key, hit, prims) && any) return true;
    return false;
}
template <bool kAny>
PT_HD __forceinline__ bool leaf4(const DeviceScene &s, int32_t ref, const pt_ray &r, float dl, float tmin, float tmax, int tie,
                                 bool &found, float &closest, long long &best_key, HitInfo &hit, uint32_t &prims) {
    return leaf4_rt(s, ref, r, dl, tmin, tmax, tie, kAny, found, closest, best_key, hit, prims);
}

// Per-thread four-wide walk (local-memory stack), for kernels that run one ray per thread;
// closest hit or any hit chosen at run time, so that lanes of one warp walking rays of both
// kinds run the same instructions.
PT_HD inline bool traverse4_rt(const DeviceScene &s, const pt_ray &r, float tmin, float tmax, int tie, bool any,
                               HitInfo &hit, uint32_t &boxes, uint32_t &prims, int &error, int32_t root = 0) {
    hit.slot = -1; hit.t = 0; hit.u = 0; hit.v = 0;
    if (s.empty || s.node_count == 0 || root < 0) return false;
    RayBox4 rb = ray_box4(r);
    float dl = length(mk(r.direction));
    bool found = false;
    float closest = tmax, limit = tmax;
    long long best_key = 0;
    int32_t sref[3 * kStackCapacity];
    float sdist[3 * kStackCapacity];
    int sp = 0;
    int32_t cur = root;
    for (;;) {
        if (cur >= 0) {
            int32_t ref[4];
            float dist[4];
            int hits = node4_children(s, cur, rb, tmin, limit, ref, dist, boxes);
            if (hits) {
                if (sp + hits - 1 > 3 * kStackCapacity) { error = 1; hit.slot = -1; return false; }
#pragma unroll
                for (int k = 3; k >= 1; k--)           // static indices: ref/dist stay in registers
                    if (k < hits) { sref[sp] = ref[k]; sdist[sp] = dist[k]; sp++; }
                cur = ref[0];
                continue;
            }
        } else {
            if (leaf4_rt(s, cur, r, dl, tmin, tmax, tie, any, found, closest, best_key, hit, prims) && any) return true;
            if (found) limit = nextafterf(closest, tmax);
        }
        // pop the nearest entry still inside the limit
        bool next = false;
        while (sp > 0) {
            sp--;
            if (sdist[sp] < limit) { cur = sref[sp]; next = true; break; }
        }
        if (!next) break;
    }
    return found;
}
template <bool kAny>
PT_HD inline bool traverse4(const DeviceScene &s, const pt_ray &r, float tmin, float tmax, int tie,
                            HitInfo &hit, uint32_t &boxes, uint32_t &prims, int &error, int32_t root = 0) {
    return traverse4_rt(s, r, tmin, tmax, tie, kAny, hit, boxes, prims, error, root);
}

} // namespace ptb

#ifdef __CUDACC__
namespace ptb {

// Four-wide form of persistent_walk (same contract).  Each lane keeps kSharedStack4 stack
// entries (reference + entry distance) in shared memory, entry-major, the rest in local memory.
constexpr int kSharedStack4 = 16;
constexpr int kStack4 = 3 * kStackCapacity;

template <bool kAny, class Get, class Done>
__device__ inline void persistent_walk4(const DeviceScene &s, size_t count, unsigned long long *next, int min_active,
                                        int tie, Get get, Done done) {
    const size_t warp_first = (size_t(blockIdx.x) * blockDim.x + (threadIdx.x & ~31u));
    if (warp_first >= count) return;
    extern __shared__ int32_t shared_stack[];
    int2 *my_stack = reinterpret_cast<int2 *>(shared_stack) + threadIdx.x;
    const int stride = blockDim.x;
    int2 spill[kStack4 - kSharedStack4];
    const unsigned lane = threadIdx.x & 31;
    pt_ray r;
    RayBox4 rb;
    float dl = 0, tmin = 0, tmax = 0, closest = 0, limit = 0;
    long long best_key = 0;
    HitInfo hit;
    uint32_t boxes = 0, prims = 0;
    int32_t cur = -1;
    int sp = 0;
    bool found = false;
    int error = 0;
    size_t index = 0;
    bool busy = false, pool_empty = false;
    hit.slot = -1; hit.t = 0; hit.u = 0; hit.v = 0;
    for (;;) {
        unsigned idle = __ballot_sync(0xffffffffu, !busy);
        if (idle && !pool_empty) {
            int leader = __ffs(idle) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(next, (unsigned long long)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(idle) >= count) pool_empty = true;
            if (!busy) {
                size_t mine = base + __popc(idle & ((1u << lane) - 1u));
                if (mine < count) {
                    index = mine;
                    get(index, r, tmin, tmax);
                    rb = ray_box4(r);
                    dl = length(mk(r.direction));
                    closest = tmax; limit = tmax; best_key = 0;
                    hit.slot = -1; hit.t = 0; hit.u = 0; hit.v = 0;
                    boxes = 0; prims = 0; sp = 0; found = false; error = 0;
                    cur = (s.empty || s.node_count == 0) ? kEmptyChild : 0;
                    busy = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, busy)) break;
        const int threshold = pool_empty ? 1 : min_active;
        for (;;) {
            if (busy) {
                bool end = cur == kEmptyChild, descended = false;
                if (!end && cur >= 0) {
                    int32_t ref[4];
                    float dist[4];
                    int hits = node4_children(s, cur, rb, tmin, limit, ref, dist, boxes);
                    if (hits) {
                        if (sp + hits - 1 > kStack4) { error = 1; found = false; end = true; }
                        else {
#pragma unroll
                            for (int k = 3; k >= 1; k--) {    // static indices: ref/dist stay in registers
                                if (k < hits) {
                                    int2 e = make_int2(ref[k], __float_as_int(dist[k]));
                                    if (sp < kSharedStack4) my_stack[sp * stride] = e; else spill[sp - kSharedStack4] = e;
                                    sp++;
                                }
                            }
                            cur = ref[0];
                            descended = true;
                        }
                    }
                } else if (!end) {
                    if (leaf4<kAny>(s, cur, r, dl, tmin, tmax, tie, found, closest, best_key, hit, prims) && kAny) end = true;
                    else if (found) limit = nextafterf(closest, tmax);
                }
                if (!end && !descended) {
                    end = true;
                    while (sp > 0) {
                        sp--;
                        int2 e = sp < kSharedStack4 ? my_stack[sp * stride] : spill[sp - kSharedStack4];
                        if (__int_as_float(e.y) < limit) { cur = e.x; end = false; break; }
                    }
                }
                if (end) {
                    WalkResult res;
                    res.t = hit.t; res.u = hit.u; res.v = hit.v; res.slot = found ? hit.slot : -1;
                    res.boxes = boxes; res.prims = prims; res.error = error;
                    done(index, res);
                    busy = false;
                    cur = kEmptyChild;
                }
            }
            if (__popc(__ballot_sync(0xffffffffu, busy)) < threshold) break;
        }
    }
}

} // namespace ptb
#endif

#ifdef __CUDACC__
namespace ptb {

// Four-wide walk in two phases per round (speculative while-while): in the node phase every
// lane walks inner nodes until it holds a postponed leaf — lanes that already hold one keep
// walking speculatively while others search, and postpone a second leaf when they reach one;
// the phase also ends once fewer than four lanes are still searching while another holds a
// leaf — and in the leaf phase all lanes test their leaves together, so node work and primitive
// work do not diverge inside one warp instruction stream.  Same contract and answer as
// persistent_walk4 (a leaf tested after a nearer hit was found only costs time: the triangle
// tests take the current closest distance as their limit).
// With kRoot, get() also returns the walk's root node (several trees in one node array; < 0 for
// an empty tree).
template <bool kAny, bool kRoot = false, class Get, class Done>
__device__ inline void persistent_walk4_spec(const DeviceScene &s, size_t count, unsigned long long *next, int min_active,
                                             int tie, Get get, Done done) {
    const size_t warp_first = (size_t(blockIdx.x) * blockDim.x + (threadIdx.x & ~31u));
    if (warp_first >= count) return;
    extern __shared__ int32_t shared_stack[];
    int2 *my_stack = reinterpret_cast<int2 *>(shared_stack) + threadIdx.x;
    const int stride = blockDim.x;
    int2 spill[kStack4 - kSharedStack4];
    const unsigned lane = threadIdx.x & 31;
    constexpr int32_t kNone = kEmptyChild;
    pt_ray r;
    RayBox4 rb;
    float dl = 0, tmin = 0, tmax = 0, closest = 0, limit = 0;
    long long best_key = 0;
    HitInfo hit;
    uint32_t boxes = 0, prims = 0;
    int32_t cur = kNone, leaf = kNone, leaf2 = kNone;
    int sp = 0;
    bool found = false;
    int error = 0;
    size_t index = 0;
    bool busy = false, pool_empty = false;
    hit.slot = -1; hit.t = 0; hit.u = 0; hit.v = 0;
    auto pop = [&]() -> int32_t {
        while (sp > 0) {
            sp--;
            int2 e = sp < kSharedStack4 ? my_stack[sp * stride] : spill[sp - kSharedStack4];
            if (__int_as_float(e.y) < limit) return e.x;
        }
        return kNone;
    };
    for (;;) {
        unsigned idle = __ballot_sync(0xffffffffu, !busy);
        if (idle && !pool_empty) {
            int leader = __ffs(idle) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(next, (unsigned long long)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(idle) >= count) pool_empty = true;
            if (!busy) {
                size_t mine = base + __popc(idle & ((1u << lane) - 1u));
                if (mine < count) {
                    index = mine;
                    int32_t root = 0;
                    if constexpr (kRoot) get(index, r, tmin, tmax, root);
                    else get(index, r, tmin, tmax);
                    rb = ray_box4(r);
                    dl = length(mk(r.direction));
                    closest = tmax; limit = tmax; best_key = 0;
                    hit.slot = -1; hit.t = 0; hit.u = 0; hit.v = 0;
                    boxes = 0; prims = 0; sp = 0; found = false; error = 0;
                    cur = (s.empty || s.node_count == 0 || root < 0) ? kNone : root;
                    leaf = kNone; leaf2 = kNone;
                    busy = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, busy)) break;
        const int threshold = pool_empty ? 1 : min_active;
        for (;;) {
            bool end = false;
            // ---- node phase: per iteration a node step, the postponement of a leaf, and at most one pop
            for (;;) {
                bool need_pop = false;
                if (busy && cur >= 0 && cur != kNone && !error) {
                    int32_t ref[4];
                    float dist[4];
                    int hits = node4_children(s, cur, rb, tmin, limit, ref, dist, boxes);
                    if (hits) {
                        if (sp + hits - 1 > kStack4) { error = 1; cur = kNone; leaf = kNone; leaf2 = kNone; }
                        else {
#pragma unroll
                            for (int k = 3; k >= 1; k--) {    // static indices: ref/dist stay in registers
                                if (k < hits) {
                                    int2 e = make_int2(ref[k], __float_as_int(dist[k]));
                                    if (sp < kSharedStack4) my_stack[sp * stride] = e; else spill[sp - kSharedStack4] = e;
                                    sp++;
                                }
                            }
                            cur = ref[0];
                        }
                    } else {
                        need_pop = true;
                    }
                }
                if (busy && cur < 0) {
                    if (leaf == kNone) { leaf = cur; need_pop = true; }
                    else if (leaf2 == kNone) { leaf2 = cur; need_pop = true; }
                }
                if (need_pop) cur = pop();
                bool searching = busy && leaf == kNone && cur != kNone;
                const unsigned sm = __ballot_sync(0xffffffffu, searching);
                if (!sm) break;
                // a few searching lanes do not hold the warp in the node phase once others have a
                // leaf to test (the leaf phase then makes progress, so no round is empty)
                if (__popc(sm) < 4 && __any_sync(0xffffffffu, busy && leaf != kNone)) break;
            }
            // ---- leaf phase
            if (busy && leaf != kNone) {
                // both postponed leaves' slots in one loop (a lane with one short leaf does not wait
                // for the warp's longest first leaf and then its longest second one)
                const int32_t v1 = ~leaf, f1 = v1 >> 3, c1 = (v1 & 7) + 1;
                int32_t f2 = 0, c2 = 0;
                if (leaf2 != kNone) { const int32_t v2 = ~leaf2; f2 = v2 >> 3; c2 = (v2 & 7) + 1; }
                for (int32_t j = 0; j < c1 + c2; j++) {
                    const int32_t slot = j < c1 ? f1 + j : f2 + (j - c1);
                    if (test_leaf<kAny>(s, slot, r, dl, tmin, tmax, tie, found, closest, best_key, hit, prims) && kAny) { end = true; break; }
                }
                if (!end && found) limit = nextafterf(closest, tmax);
                leaf = kNone; leaf2 = kNone;
            }
            if (busy && (end || error || (leaf == kNone && cur == kNone))) {
                WalkResult res;
                if (error) found = false;
                res.t = hit.t; res.u = hit.u; res.v = hit.v; res.slot = found ? hit.slot : -1;
                res.boxes = boxes; res.prims = prims; res.error = error;
                done(index, res);
                busy = false;
                cur = kNone; leaf = kNone; leaf2 = kNone;
            }
            if (__popc(__ballot_sync(0xffffffffu, busy)) < threshold) break;
        }
    }
}

} // namespace ptb
#endif
