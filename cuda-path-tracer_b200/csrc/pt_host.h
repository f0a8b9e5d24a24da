// pt_host.h — host-side pieces of the path-tracing core (validation, emitter table,
// BVH re-layout, SAH builder, workload generators).  Internal; the C ABI is include/pt.h.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>
#include "pt_internal.h"

namespace ptb {

// Error carrying a pt_status, turned into a return code at the C boundary.
struct Error : std::runtime_error {
    pt_status status;
    Error(pt_status s, const std::string &what) : std::runtime_error(what), status(s) {}
};

// validate_flat_scene (src/flat/flat_validate.h:10-83); throws Error(PT_INVALID_SCENE).
void validate_scene(const pt_scene_desc &scene);
// scene_lights (src/renderer/scene_view.h:10-28); throws Error(PT_INVALID_ARGUMENT).
std::vector<pt_light> scene_lights(const pt_scene_desc &scene, float &total_area);

// Device layout of a validated scene, built on the host.
struct HostLayout {
    std::vector<BvhNode> nodes;
    std::vector<TriRecord> tris;
    std::vector<SphereRecord> spheres;
    std::vector<int32_t> brute_order;   // leaf slots in flat node-array order
    int32_t empty = 1;
    float root_lo[3] = {0, 0, 0}, root_hi[3] = {0, 0, 0};
    int32_t root_leaf = 0;
    std::vector<Bvh4Node> nodes4;       // empty when the flat graph shares subtrees
    std::vector<Bvh4QNode> nodes4q;     // nodes4 quantized (what the device walks)
};
HostLayout relayout(const pt_scene_desc &scene);
Bvh4QNode quantize4(const Bvh4Node &n);

// Host-owned flattened scene (what the reference keeps in flat_scene).
struct FlatScene {
    std::vector<pt_triangle> triangles;
    std::vector<pt_sphere> spheres;
    std::vector<pt_node> nodes;
    std::vector<pt_material> materials;
    std::vector<pt_texture> textures;
    std::vector<unsigned char> pixels;
    int32_t root = -1;
    int32_t max_depth = 0;
    pt_scene_desc desc() const;
};

// Binned-SAH BVH over the scene's primitives, one primitive per leaf, exported in
// depth-first preorder with the reference's bounds (padded triangle boxes,
// src/geometry/triangle.h:96-109; sphere boxes center +/- r, src/geometry/sphere.h:67-73;
// branch boxes = surrounding_box, src/bvh/aabb.h:41-55).  Triangle and sphere arrays keep
// their order, so primitive ids are the caller's indices.
void build_sah(FlatScene &scene, int threads);

// Builder interchange: primitive bounds (the reference's padded triangle boxes, sphere boxes),
// temporary nodes (children are indices into the same array) and the preorder export both
// builders share (one primitive per leaf, depth <= 64).
struct BuildPrim { float lo[3], hi[3]; int32_t type, id; };
struct BuildNode { float lo[3], hi[3]; int32_t left, right, type, prim; };
std::vector<BuildPrim> gather_prims(const FlatScene &scene);
void export_preorder(FlatScene &scene, const std::vector<BuildNode> &nodes, int32_t root);
// Binned-SAH binary tree over arbitrary boxes (one per leaf; a leaf keeps its item's type and id);
// `root` receives the root's index.  threads <= 0: all.
std::vector<BuildNode> sah_tree(const std::vector<BuildPrim> &items, int threads, int32_t &root);
// Linear BVH on the GPU (pt_lbvh.cu): Morton order of centroids, Karras's radix tree.
void build_lbvh(FlatScene &scene);

int hardware_threads();

} // namespace ptb

// The C ABI's host-owned flat scene handle (include/pt_workloads.h).
struct pt_flat { ptb::FlatScene scene; };
