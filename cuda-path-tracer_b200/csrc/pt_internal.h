// pt_internal.h — device-side layouts of the B200 path-tracing core (shared host/device).
//
// HBM layout of a scene (all arrays 16-byte aligned, read with 16-byte vector loads):
//   nodes    : one 64-byte record per branch of the caller's flattened BVH, holding the
//              boxes of BOTH children (two-child "boxes in the parent" layout), so one
//              node fetch answers two box tests.
//   tris     : one 48-byte record per triangle leaf, {v0, eps}, {e1, id}, {e2, -}, where
//              e1 = v1-v0, e2 = v2-v0 and eps = 1e-7f*|e1 x e2| are computed on the host
//              with the same FP32 operations the reference performs per test
//              (src/flat/flat_intersect.h:10-18), so the device test is bit-identical.
//   spheres  : one 32-byte record per sphere leaf {center, radius}, {id, -, -, -}.
//   shading  : the caller's flat_triangle / flat_sphere / flat_material / flat_texture
//              arrays, untouched, read only for the winning hit of a ray.
#pragma once

#include <cstdint>
#include "../../include/pt.h"

#ifdef __CUDACC__
#define PT_HD __host__ __device__
#else
#define PT_HD
#endif

namespace ptb {

// Child reference: >= 0 internal node; < 0 leaf slot ~child.  Slots [0, tri_slots) are
// triangles, [tri_slots, tri_slots + sphere_slots) spheres.
constexpr int32_t kEmptyChild = 0x7fffffff;
constexpr int kStackCapacity = 64;   // flat_stack_capacity, src/flat/flat_data.h:52

struct alignas(16) BvhNode {
    // child 0 box x/y, child 1 box x/y, both boxes' z, children
    float c0lox, c0hix, c0loy, c0hiy;
    float c1lox, c1hix, c1loy, c1hiy;
    float c0loz, c0hiz, c1loz, c1hiz;
    int32_t child0, child1, pad0, pad1;
};
static_assert(sizeof(BvhNode) == 64, "node is 64 bytes");

// Four-wide node collapsed from the binary tree: the boxes of up to four children in SoA
// (x/y/z min and max, four lanes each) and their references.  A child reference >= 0 is another
// four-wide node; < 0 is a leaf of 1..8 consecutive slots, ~(first_slot << 3 | (count - 1));
// kEmptyChild marks an unused lane (its box is inverted, so it never passes).  This is the form
// the host builds; the device walks it quantized (Bvh4QNode).
struct alignas(16) Bvh4Node {
    float lox[4], hix[4], loy[4], hiy[4], loz[4], hiz[4];
    int32_t child[4];
};
static_assert(sizeof(Bvh4Node) == 112, "four-wide node is 112 bytes");
constexpr int kLeafMax = 4;   // slots per four-wide leaf

// Quantized four-wide node (64 bytes, half a cache line, two 32-byte loads): the children's boxes
// on a per-axis power-of-two grid anchored at the low corner (px, py, pz) of their union, 8 bits
// per bound, lower bounds rounded down and upper bounds up, so a dequantised box (p + q * 2^e)
// always contains the child's true box.  The grid spacing is the smallest power of two with 255
// steps covering the union.  An empty slot has its lower bounds above its upper ones.
struct alignas(64) Bvh4QNode {
    float px, py, pz;
    float sx;                      // grid spacing along x (a power of two)
    uint32_t qlo[3], qhi[3];       // per axis; child k in byte k
    int32_t child[4];
    float sy, sz;                  // grid spacings along y and z
};
static_assert(sizeof(Bvh4QNode) == 64, "quantized four-wide node is 64 bytes");

struct alignas(16) TriRecord {
    float v0x, v0y, v0z, eps;
    float e1x, e1y, e1z; int32_t id;
    float e2x, e2y, e2z; int32_t node;   // flat node index of the leaf (reference tie order)
};
static_assert(sizeof(TriRecord) == 48, "triangle record is 48 bytes");

struct alignas(16) SphereRecord {
    float cx, cy, cz, radius;
    int32_t id, node, pad0, pad1;
};
static_assert(sizeof(SphereRecord) == 32, "sphere record is 32 bytes");

// Everything a kernel needs, passed by value (device pointers).
struct DeviceScene {
    const BvhNode *nodes;
    const Bvh4QNode *nodes4;        // null when the tree could not be collapsed (shared subtrees)
    const TriRecord *tris;
    const SphereRecord *spheres;
    const pt_triangle *triangles;   // caller's records (shading, light sampling)
    const pt_sphere *sphere_src;
    const pt_material *materials;
    const pt_texture *textures;
    const unsigned char *pixels;
    const pt_light *lights;
    int32_t node_count;             // internal nodes (0 for an empty scene)
    int32_t tri_slots, sphere_slots;
    int32_t light_count;
    float light_area;
    int32_t empty;                  // root == -1
    float root_lo[3], root_hi[3];   // the flat root's own box (tested first by trace_world)
    int32_t root_leaf;              // flat root is itself a leaf (no branch above it)
};

// Tie rule for exact-distance hits: the lowest (type, id) (the parity rule of the query API), the leaf the
// reference's depth-first walk reaches last (trace_world, src/renderer/transport.h:76-79), or
// the last leaf in node-array order (its brute-force scan, transport.h:48-60).
enum TieRule : int { kTieLowestId = 0, kTieLastLeaf = 1, kTieLastNode = 2 };

} // namespace ptb
