// pt_lbvh.cu — BVH construction on the GPU (linear BVH).
//
// Replaces the host build that produces the flattened arrays (the reference's bvh_node,
// src/bvh/bvh.h:132-171, and this library's binned SAH, pt_build.cpp) for scenes that must be
// built fast: primitives are ordered along a 63-bit Morton curve of their box centroids (21 bits
// per axis over the centroid bounds), and the binary radix tree over the sorted codes is built
// with every internal node in parallel (Karras, "Maximizing Parallelism in the Construction of
// BVHs, Octrees, and k-d Trees", HPG 2012; equal codes are told apart by their sorted index).
// Boxes are unions of the children's, computed bottom-up (a node's second arriving child
// computes it), so every node box encloses the reference's padded primitive boxes exactly.
// The tree is exported on the host with the same preorder as the SAH builder (one primitive per
// leaf, depth <= 64).  Tree quality is that of a linear BVH: traversal is somewhat slower than
// on the SAH tree; the build is much faster.
#include <cub/device/device_radix_sort.cuh>
#include <algorithm>
#include <cfloat>
#include <vector>
#include "pt_api_common.h"
#include "pt_device.h"
#include "../../include/pt_workloads.h"

using namespace ptb;

namespace ptb {
namespace lbvh {

struct Bounds { float lo[3], hi[3]; };

__device__ inline uint64_t spread21(uint64_t x) {   // bit k of x -> bit 3k
    x &= 0x1fffff;
    x = (x | (x << 32)) & 0x1f00000000ffffull;
    x = (x | (x << 16)) & 0x1f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// centroid bounds: a warp reduction, then one atomic per warp on an order-preserving unsigned
// image of the float (negative values bit-inverted, positive ones with the sign bit set)
__device__ inline unsigned int ordered(float f) {
    unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ inline float unordered(unsigned int u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void centroid_bounds(const BuildPrim *prims, int n, unsigned int *bounds /* 6: min xyz, max xyz */) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < n;
    for (int a = 0; a < 3; a++) {
        unsigned int mn = 0xffffffffu, mx = 0u;
        if (valid) mn = mx = ordered(0.5f * (prims[i].lo[a] + prims[i].hi[a]));
        for (int o = 16; o; o >>= 1) {       // warp reduction, then one atomic per warp
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        if ((threadIdx.x & 31) == 0) { atomicMin(&bounds[a], mn); atomicMax(&bounds[3 + a], mx); }
    }
}

__global__ void morton_codes(const BuildPrim *prims, int n, const unsigned int *bounds, uint64_t *codes, int32_t *order) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t q[3];
    for (int a = 0; a < 3; a++) {
        float lo = unordered(bounds[a]), hi = unordered(bounds[3 + a]);
        float c = 0.5f * (prims[i].lo[a] + prims[i].hi[a]);
        float extent = hi - lo;
        float t = extent > 0 ? (c - lo) / extent : 0.0f;
        t = fminf(fmaxf(t, 0.0f), 1.0f);
        q[a] = uint64_t(fminf(t * 2097152.0f, 2097151.0f));
    }
    codes[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    order[i] = i;
}

// length of the common prefix of sorted keys i and j (index bits break ties); -1 outside
__device__ inline int delta(const uint64_t *k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint64_t a = k[i], b = k[j];
    if (a == b) return 64 + __clz(unsigned(i) ^ unsigned(j));
    return __clzll(a ^ b);
}

// Internal node i of n - 1: its key range, split and children.  Children are encoded as
// internal index (>= 0) or ~leaf index (< 0).
__global__ void radix_tree(const uint64_t *k, int n, int32_t *left, int32_t *right, int32_t *parent_internal,
                           int32_t *parent_leaf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = delta(k, n, i, i + 1) - delta(k, n, i, i - 1) >= 0 ? 1 : -1;
    int dmin = delta(k, n, i, i - d);
    int lmax = 2;
    while (delta(k, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(k, n, i, j);
    int s = 0;
    for (int div = 2;; div *= 2) {
        int t = (l + div - 1) / div;
        if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
    }
    int g = i + s * d + min(d, 0);
    int lo = min(i, j), hi = max(i, j);
    int32_t lc = lo == g ? ~g : g;
    int32_t rc = hi == g + 1 ? ~(g + 1) : g + 1;
    left[i] = lc;
    right[i] = rc;
    if (lc < 0) parent_leaf[~lc] = i; else parent_internal[lc] = i;
    if (rc < 0) parent_leaf[~rc] = i; else parent_internal[rc] = i;
}

// Bottom-up boxes: each leaf climbs; at every node the first arriving child stops, the second
// unions both children's boxes and climbs on.
__global__ void refit(const BuildPrim *prims, const int32_t *order, int n, const int32_t *left, const int32_t *right,
                      const int32_t *parent_internal, const int32_t *parent_leaf, unsigned int *arrivals, Bounds *boxes) {
    int leaf = blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= n) return;
    int node = parent_leaf[leaf];
    while (node >= 0) {
        __threadfence();
        if (atomicAdd(&arrivals[node], 1u) == 0) return;
        __threadfence();
        Bounds b;
        for (int a = 0; a < 3; a++) { b.lo[a] = FLT_MAX; b.hi[a] = -FLT_MAX; }
        const int32_t kids[2] = {left[node], right[node]};
        for (int c = 0; c < 2; c++) {
            int32_t kid = kids[c];
            if (kid < 0) {
                const BuildPrim &p = prims[order[~kid]];
                for (int a = 0; a < 3; a++) { b.lo[a] = fminf(b.lo[a], p.lo[a]); b.hi[a] = fmaxf(b.hi[a], p.hi[a]); }
            } else {
                const volatile Bounds &q = boxes[kid];
                for (int a = 0; a < 3; a++) { b.lo[a] = fminf(b.lo[a], q.lo[a]); b.hi[a] = fmaxf(b.hi[a], q.hi[a]); }
            }
        }
        boxes[node] = b;
        node = parent_internal[node];
    }
}

} // namespace lbvh

void build_lbvh(FlatScene &scene) {
    using namespace lbvh;
    std::vector<BuildPrim> prims = gather_prims(scene);
    const int n = int(prims.size());
    if (n <= 1) {
        std::vector<BuildNode> nodes;
        if (n == 1) {
            BuildNode leaf{};
            for (int a = 0; a < 3; a++) { leaf.lo[a] = prims[0].lo[a]; leaf.hi[a] = prims[0].hi[a]; }
            leaf.left = leaf.right = -1; leaf.type = prims[0].type; leaf.prim = prims[0].id;
            nodes.push_back(leaf);
        }
        export_preorder(scene, nodes, n == 1 ? 0 : -1);
        return;
    }
    require_device();
    DeviceBuffer d_prims, d_bounds, d_codes, d_codes_sorted, d_order, d_order_sorted, d_left, d_right, d_pi, d_pl, d_arr, d_boxes, d_temp;
    d_prims.upload(prims);
    const unsigned int init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    d_bounds.upload(init, sizeof init);
    d_codes.resize(size_t(n) * 8); d_codes_sorted.resize(size_t(n) * 8);
    d_order.resize(size_t(n) * 4); d_order_sorted.resize(size_t(n) * 4);
    d_left.resize(size_t(n - 1) * 4); d_right.resize(size_t(n - 1) * 4);
    d_pi.resize(size_t(n - 1) * 4); d_pl.resize(size_t(n) * 4);
    d_arr.resize(size_t(n - 1) * 4); d_boxes.resize(size_t(n - 1) * sizeof(Bounds));
    PT_CUDA(cudaMemset(d_arr.get(), 0, size_t(n - 1) * 4));
    PT_CUDA(cudaMemset(d_pi.get(), 0xff, size_t(n - 1) * 4));    // root's parent = -1
    const int blocks = (n + 255) / 256;
    centroid_bounds<<<blocks, 256>>>(d_prims.get<BuildPrim>(), n, d_bounds.get<unsigned int>());
    morton_codes<<<blocks, 256>>>(d_prims.get<BuildPrim>(), n, d_bounds.get<unsigned int>(), d_codes.get<uint64_t>(), d_order.get<int32_t>());
    PT_CUDA(cudaGetLastError());
    size_t temp = 0;
    PT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, d_codes.get<uint64_t>(), d_codes_sorted.get<uint64_t>(),
                                            d_order.get<int32_t>(), d_order_sorted.get<int32_t>(), n, 0, 63));
    d_temp.resize(std::max<size_t>(temp, 1));
    PT_CUDA(cub::DeviceRadixSort::SortPairs(d_temp.get(), temp, d_codes.get<uint64_t>(), d_codes_sorted.get<uint64_t>(),
                                            d_order.get<int32_t>(), d_order_sorted.get<int32_t>(), n, 0, 63));
    radix_tree<<<(n - 1 + 255) / 256, 256>>>(d_codes_sorted.get<uint64_t>(), n, d_left.get<int32_t>(), d_right.get<int32_t>(),
                                              d_pi.get<int32_t>(), d_pl.get<int32_t>());
    refit<<<blocks, 256>>>(d_prims.get<BuildPrim>(), d_order_sorted.get<int32_t>(), n, d_left.get<int32_t>(), d_right.get<int32_t>(),
                           d_pi.get<int32_t>(), d_pl.get<int32_t>(), d_arr.get<unsigned int>(), d_boxes.get<Bounds>());
    PT_CUDA(cudaGetLastError());
    std::vector<int32_t> left(size_t(n - 1)), right(size_t(n - 1)), order(static_cast<size_t>(n));
    std::vector<Bounds> boxes(size_t(n - 1));
    PT_CUDA(cudaMemcpy(left.data(), d_left.get(), left.size() * 4, cudaMemcpyDeviceToHost));
    PT_CUDA(cudaMemcpy(right.data(), d_right.get(), right.size() * 4, cudaMemcpyDeviceToHost));
    PT_CUDA(cudaMemcpy(order.data(), d_order_sorted.get(), order.size() * 4, cudaMemcpyDeviceToHost));
    PT_CUDA(cudaMemcpy(boxes.data(), d_boxes.get(), boxes.size() * sizeof(Bounds), cudaMemcpyDeviceToHost));
    // nodes: internal 0..n-2, then leaf k at n-1+k
    std::vector<BuildNode> nodes(size_t(2 * n - 1));
    auto child = [&](int32_t c) { return c < 0 ? int32_t(n - 1 + ~c) : c; };
    for (int i = 0; i < n - 1; i++) {
        BuildNode &b = nodes[size_t(i)];
        for (int a = 0; a < 3; a++) { b.lo[a] = boxes[size_t(i)].lo[a]; b.hi[a] = boxes[size_t(i)].hi[a]; }
        b.left = child(left[size_t(i)]); b.right = child(right[size_t(i)]); b.type = PT_BRANCH; b.prim = -1;
    }
    for (int k = 0; k < n; k++) {
        const BuildPrim &p = prims[size_t(order[size_t(k)])];
        BuildNode &b = nodes[size_t(n - 1 + k)];
        for (int a = 0; a < 3; a++) { b.lo[a] = p.lo[a]; b.hi[a] = p.hi[a]; }
        b.left = b.right = -1; b.type = p.type; b.prim = p.id;
    }
    export_preorder(scene, nodes, 0);
}

} // namespace ptb

extern "C" pt_status pt_flat_build_bvh_gpu(pt_flat *scene) {
    return guard([&]() {
        if (!scene) throw Error(PT_INVALID_ARGUMENT, "null scene");
        build_lbvh(scene->scene);
    });
}
