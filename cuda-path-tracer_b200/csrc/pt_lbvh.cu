// pt_lbvh.cu — BVH construction on the GPU (Morton order, agglomerative clustering, SAH top).
//
// Replaces the host build that produces the flattened arrays (the reference's bvh_node,
// src/bvh/bvh.h:132-171, and this library's binned SAH, pt_build.cpp) for scenes that must be
// built fast.  Three stages:
//   1. primitives are ordered along a 63-bit Morton curve of their box centroids (21 bits per
//      axis over the centroid bounds; a radix sort on the device);
//   2. locally-ordered clustering on the device (Meister and Bittner, "Parallel Locally-Ordered
//      Clustering for Bounding Volume Hierarchy Construction", 2018): in every round each cluster
//      finds, among the clusters up to kRadius places away in Morton order, the one whose union
//      with it has the smallest surface area (ties: the lower index, so pairs are totally
//      ordered and the best pair is always mutual); mutual nearest neighbours merge into a new
//      node at the lower index, and the clusters are compacted in order.  Rounds run until a
//      quarter of the primitives' count remains (each cluster then holds a few primitives);
//   3. the binned-SAH builder of pt_build.cpp splits the remaining cluster boxes on the host, and
//      the clusters' subtrees hang under its leaves.
// Boxes are unions of the children's, so every node box encloses the reference's padded
// primitive boxes exactly.  The tree is exported with the SAH builder's preorder (one primitive
// per leaf, depth <= 64).  Merging by nearest neighbour makes the lowest levels a little worse
// than SAH splits: the tree traverses a few percent slower than the host SAH tree.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
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

constexpr int kRadius = 16;         // neighbours searched on each side, in Morton order
constexpr int kNearBlock = 256;

__device__ inline float merged_area(const Bounds &a, const Bounds &b) {
    float dx = fmaxf(a.hi[0], b.hi[0]) - fminf(a.lo[0], b.lo[0]);
    float dy = fmaxf(a.hi[1], b.hi[1]) - fminf(a.lo[1], b.lo[1]);
    float dz = fmaxf(a.hi[2], b.hi[2]) - fminf(a.lo[2], b.lo[2]);
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

// leaf k (k-th primitive in Morton order) is node k; every leaf starts as its own cluster
__global__ void leaf_boxes(const BuildPrim *prims, const int32_t *order, int n, Bounds *boxes, int32_t *clusters) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const BuildPrim &p = prims[order[k]];
    Bounds b;
    for (int a = 0; a < 3; a++) { b.lo[a] = p.lo[a]; b.hi[a] = p.hi[a]; }
    boxes[k] = b;
    clusters[k] = k;
}

// nearest neighbour of every cluster within kRadius places (smallest merged area, then lowest index)
__global__ void __launch_bounds__(kNearBlock) nearest(const Bounds *boxes, const int32_t *clusters, int count, int32_t *nn) {
    __shared__ Bounds tile[kNearBlock + 2 * kRadius];
    const int base = blockIdx.x * kNearBlock;
    for (int t = threadIdx.x; t < kNearBlock + 2 * kRadius; t += kNearBlock) {
        int j = base - kRadius + t;
        if (j >= 0 && j < count) tile[t] = boxes[clusters[j]];
    }
    __syncthreads();
    const int i = base + threadIdx.x;
    if (i >= count) return;
    const Bounds bi = tile[threadIdx.x + kRadius];
    float best = FLT_MAX;
    int32_t bj = -1;
    for (int d = -kRadius; d <= kRadius; d++) {
        const int j = i + d;
        if (d == 0 || j < 0 || j >= count) continue;
        const float area = merged_area(bi, tile[threadIdx.x + kRadius + d]);
        if (area < best) { best = area; bj = j; }
    }
    nn[i] = bj;
}

// merge[i] = 1 when cluster i is the lower index of a mutual pair; keep[i] = 0 for the upper one
__global__ void pair_flags(const int32_t *nn, int count, int32_t *merge, unsigned char *keep) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int32_t j = nn[i];
    const bool mutual = j >= 0 && nn[j] == i;
    merge[i] = mutual && i < j;
    keep[i] = !(mutual && i > j);
}

// the lower cluster of each mutual pair becomes a new node (numbered by the pairs' scan)
__global__ void merge_pairs(const int32_t *clusters, const int32_t *nn, const int32_t *merge, const int32_t *slot, int count,
                            int32_t node_base, Bounds *boxes, int32_t *left, int32_t *right, int32_t *merged) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    if (!merge[i]) { merged[i] = clusters[i]; return; }
    const int32_t a = clusters[i], b = clusters[nn[i]], id = node_base + slot[i];
    Bounds u;
    const Bounds ba = boxes[a], bb = boxes[b];
    for (int k = 0; k < 3; k++) { u.lo[k] = fminf(ba.lo[k], bb.lo[k]); u.hi[k] = fmaxf(ba.hi[k], bb.hi[k]); }
    boxes[id] = u;
    left[id] = a;
    right[id] = b;
    merged[i] = id;
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
    // node ids: leaf k = k (Morton order), merged nodes from n upwards (at most n - 1 of them)
    const size_t total = size_t(2 * n - 1);
    DeviceBuffer d_prims, d_bounds, d_codes, d_codes_sorted, d_order, d_order_sorted, d_boxes, d_left, d_right, d_clusters,
        d_merged, d_nn, d_merge, d_slot, d_keep, d_count, d_temp;
    d_prims.upload(prims);
    const unsigned int init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    d_bounds.upload(init, sizeof init);
    d_codes.resize(size_t(n) * 8); d_codes_sorted.resize(size_t(n) * 8);
    d_order.resize(size_t(n) * 4); d_order_sorted.resize(size_t(n) * 4);
    d_boxes.resize(total * sizeof(Bounds));
    d_left.resize(total * 4); d_right.resize(total * 4);
    d_clusters.resize(size_t(n) * 4); d_merged.resize(size_t(n) * 4); d_nn.resize(size_t(n) * 4);
    d_merge.resize(size_t(n) * 4); d_slot.resize(size_t(n) * 4); d_keep.resize(size_t(n)); d_count.resize(2 * sizeof(int32_t));
    const int blocks = (n + 255) / 256;
    centroid_bounds<<<blocks, 256>>>(d_prims.get<BuildPrim>(), n, d_bounds.get<unsigned int>());
    morton_codes<<<blocks, 256>>>(d_prims.get<BuildPrim>(), n, d_bounds.get<unsigned int>(), d_codes.get<uint64_t>(), d_order.get<int32_t>());
    PT_CUDA(cudaGetLastError());
    size_t sort_temp = 0, scan_temp = 0, select_temp = 0;
    PT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_temp, d_codes.get<uint64_t>(), d_codes_sorted.get<uint64_t>(),
                                            d_order.get<int32_t>(), d_order_sorted.get<int32_t>(), n, 0, 63));
    PT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_temp, d_merge.get<int32_t>(), d_slot.get<int32_t>(), n));
    PT_CUDA(cub::DeviceSelect::Flagged(nullptr, select_temp, d_merged.get<int32_t>(), d_keep.get<unsigned char>(),
                                       d_clusters.get<int32_t>(), d_count.get<int32_t>(), n));
    d_temp.resize(std::max<size_t>({sort_temp, scan_temp, select_temp, 1}));
    PT_CUDA(cub::DeviceRadixSort::SortPairs(d_temp.get(), sort_temp, d_codes.get<uint64_t>(), d_codes_sorted.get<uint64_t>(),
                                            d_order.get<int32_t>(), d_order_sorted.get<int32_t>(), n, 0, 63));
    leaf_boxes<<<blocks, 256>>>(d_prims.get<BuildPrim>(), d_order_sorted.get<int32_t>(), n, d_boxes.get<Bounds>(),
                                d_clusters.get<int32_t>());
    PT_CUDA(cudaGetLastError());
    // clustering rounds until a quarter of the primitives' count remains
    const int stop = std::max(1, n / 4);
    int count = n;
    int32_t next = n;
    for (int round = 0; count > stop; round++) {
        if (round > 4 * n) throw Error(PT_INVALID_ARGUMENT, "clustering did not converge");
        const int cb = (count + 255) / 256;
        nearest<<<(count + kNearBlock - 1) / kNearBlock, kNearBlock>>>(d_boxes.get<Bounds>(), d_clusters.get<int32_t>(), count,
                                                                     d_nn.get<int32_t>());
        pair_flags<<<cb, 256>>>(d_nn.get<int32_t>(), count, d_merge.get<int32_t>(), d_keep.get<unsigned char>());
        PT_CUDA(cudaGetLastError());
        PT_CUDA(cub::DeviceScan::ExclusiveSum(d_temp.get(), scan_temp, d_merge.get<int32_t>(), d_slot.get<int32_t>(), count));
        merge_pairs<<<cb, 256>>>(d_clusters.get<int32_t>(), d_nn.get<int32_t>(), d_merge.get<int32_t>(), d_slot.get<int32_t>(), count,
                                 next, d_boxes.get<Bounds>(), d_left.get<int32_t>(), d_right.get<int32_t>(), d_merged.get<int32_t>());
        PT_CUDA(cudaGetLastError());
        PT_CUDA(cub::DeviceSelect::Flagged(d_temp.get(), select_temp, d_merged.get<int32_t>(), d_keep.get<unsigned char>(),
                                           d_clusters.get<int32_t>(), d_count.get<int32_t>(), count));
        int32_t remaining = 0;
        PT_CUDA(cudaMemcpy(&remaining, d_count.get(), sizeof remaining, cudaMemcpyDeviceToHost));
        next += count - remaining;     // one new node per merged pair
        count = remaining;
    }
    std::vector<int32_t> left(total, -1), right(total, -1), clusters(static_cast<size_t>(count)), order(static_cast<size_t>(n));
    std::vector<Bounds> boxes(total);
    PT_CUDA(cudaMemcpy(left.data() + n, d_left.get<int32_t>() + n, size_t(next - n) * 4, cudaMemcpyDeviceToHost));
    PT_CUDA(cudaMemcpy(right.data() + n, d_right.get<int32_t>() + n, size_t(next - n) * 4, cudaMemcpyDeviceToHost));
    PT_CUDA(cudaMemcpy(boxes.data(), d_boxes.get(), size_t(next) * sizeof(Bounds), cudaMemcpyDeviceToHost));
    PT_CUDA(cudaMemcpy(clusters.data(), d_clusters.get(), size_t(count) * 4, cudaMemcpyDeviceToHost));
    PT_CUDA(cudaMemcpy(order.data(), d_order_sorted.get(), order.size() * 4, cudaMemcpyDeviceToHost));
    std::vector<BuildNode> nodes(total);
    for (int k = 0; k < n; k++) {
        const BuildPrim &p = prims[size_t(order[size_t(k)])];
        BuildNode &b = nodes[size_t(k)];
        for (int a = 0; a < 3; a++) { b.lo[a] = p.lo[a]; b.hi[a] = p.hi[a]; }
        b.left = b.right = -1; b.type = p.type; b.prim = p.id;
    }
    for (int32_t id = n; id < next; id++) {
        BuildNode &b = nodes[size_t(id)];
        for (int a = 0; a < 3; a++) { b.lo[a] = boxes[size_t(id)].lo[a]; b.hi[a] = boxes[size_t(id)].hi[a]; }
        b.left = left[size_t(id)]; b.right = right[size_t(id)]; b.type = PT_BRANCH; b.prim = -1;
    }
    int32_t root = clusters[0];
    if (count > 1) {
        // binned SAH over the remaining clusters' boxes; the clusters hang under its leaves
        std::vector<BuildPrim> items(static_cast<size_t>(count));
        for (int i = 0; i < count; i++) {
            const BuildNode &c = nodes[size_t(clusters[size_t(i)])];
            for (int a = 0; a < 3; a++) { items[size_t(i)].lo[a] = c.lo[a]; items[size_t(i)].hi[a] = c.hi[a]; }
            items[size_t(i)].type = PT_TRIANGLE;
            items[size_t(i)].id = clusters[size_t(i)];
        }
        int32_t top_root = -1;
        std::vector<BuildNode> top = sah_tree(items, 0, top_root);
        std::vector<int32_t> id_of(top.size());
        for (size_t k = 0; k < top.size(); k++) id_of[k] = top[k].type == PT_BRANCH ? next++ : top[k].prim;
        for (size_t k = 0; k < top.size(); k++) {
            if (top[k].type != PT_BRANCH) continue;
            BuildNode &b = nodes[size_t(id_of[k])];
            b = top[k];
            b.left = id_of[size_t(top[k].left)];
            b.right = id_of[size_t(top[k].right)];
        }
        root = id_of[size_t(top_root)];
    }
    export_preorder(scene, nodes, root);
}

} // namespace ptb

extern "C" pt_status pt_flat_build_bvh_gpu(pt_flat *scene) {
    return guard([&]() {
        if (!scene) throw Error(PT_INVALID_ARGUMENT, "null scene");
        build_lbvh(scene->scene);
    });
}
