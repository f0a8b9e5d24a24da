// pt_build.cpp — host binned-SAH BVH builder producing the reference's flat format.
//
// The reference builds its tree with a random axis and a median split (src/bvh/bvh.h:132-171)
// and exports it depth-first (src/flat/flat_export.h:85-123).  This builder keeps the output
// format (one primitive per leaf, preorder node array, padded triangle bounds, depth <= 64)
// and replaces the split choice with a 32-bin surface-area heuristic, built in parallel.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <future>
#include <limits>
#include "pt_host.h"

namespace ptb {
namespace {

struct Box {
    float lo[3], hi[3];
    void reset() { for(int a = 0; a < 3; a++) { lo[a] = FLT_MAX; hi[a] = -FLT_MAX; } }
    void grow(const Box &b) {
        for(int a = 0; a < 3; a++) { lo[a] = b.lo[a] < lo[a] ? b.lo[a] : lo[a]; hi[a] = b.hi[a] > hi[a] ? b.hi[a] : hi[a]; }
    }
    void grow(const float *p) {
        for(int a = 0; a < 3; a++) { lo[a] = p[a] < lo[a] ? p[a] : lo[a]; hi[a] = p[a] > hi[a] ? p[a] : hi[a]; }
    }
    double area() const {
        double d[3];
        for(int a = 0; a < 3; a++) d[a] = hi[a] > lo[a] ? double(hi[a]) - lo[a] : 0.0;
        return 2.0*(d[0]*d[1] + d[1]*d[2] + d[2]*d[0]);
    }
};

struct Prim {
    Box box;
    float centroid[3];
    int32_t type, id;
};

struct TNode {
    Box box;
    int32_t left = -1, right = -1;    // temp node ids for branches
    int32_t type = PT_BRANCH, prim = -1;
};

// triangle::bounding_box (src/geometry/triangle.h:96-109): min/max per axis, then
// nextafter(min - 0.0001f, -inf) and nextafter(max + 0.0001f, +inf).
Box triangle_box(const pt_triangle &t) {
    Box b;
    const float *v0 = &t.v0.x, *v1 = &t.v1.x, *v2 = &t.v2.x;
    const float inf = std::numeric_limits<float>::infinity();
    for(int a = 0; a < 3; a++) {
        float mn = v1[a] < v2[a] ? v1[a] : v2[a];
        mn = v0[a] < mn ? v0[a] : mn;
        float mx = v1[a] > v2[a] ? v1[a] : v2[a];
        mx = v0[a] > mx ? v0[a] : mx;
        b.lo[a] = std::nextafter(mn - 0.0001f, -inf);
        b.hi[a] = std::nextafter(mx + 0.0001f, inf);
    }
    return b;
}
// sphere::bounding_box (src/geometry/sphere.h:67-73)
Box sphere_box(const pt_sphere &s) {
    Box b;
    const float *c = &s.center.x;
    for(int a = 0; a < 3; a++) { b.lo[a] = c[a] - s.radius; b.hi[a] = c[a] + s.radius; }
    return b;
}

class Builder {
public:
    Builder(std::vector<Prim> &prims, int threads) : prims_(prims), threads_(threads) {
        nodes_.resize(prims.size() ? 2*prims.size() - 1 : 0);
    }
    int32_t run() {
        if(prims_.empty()) return -1;
        int par = 0;
        while((1 << par) < threads_ * 4) par++;
        return build(0, int32_t(prims_.size()), 1, par);
    }
    std::vector<TNode> nodes_;

private:
    static constexpr int kBins = 32;
    static constexpr int kMedianDepth = 40;   // below this depth split at the median: depth stays <= 64
    std::vector<Prim> &prims_;
    int threads_;
    std::atomic<int32_t> next_{0};

    int32_t alloc() { return next_.fetch_add(1); }

    int32_t build(int32_t begin, int32_t end, int depth, int par) {
        int32_t id = alloc();
        TNode &node = nodes_[size_t(id)];
        if(end - begin == 1) {
            node.box = prims_[size_t(begin)].box;
            node.type = prims_[size_t(begin)].type;
            node.prim = prims_[size_t(begin)].id;
            return id;
        }
        Box cb; cb.reset();
        for(int32_t i = begin; i < end; i++) cb.grow(prims_[size_t(i)].centroid);
        int32_t mid = split(begin, end, cb, depth);
        int32_t left, right;
        if(par > 0 && end - begin > 4096) {
            auto fut = std::async(std::launch::async, [&]() { return build(begin, mid, depth + 1, par - 1); });
            right = build(mid, end, depth + 1, par - 1);
            left = fut.get();
        } else {
            left = build(begin, mid, depth + 1, 0);
            right = build(mid, end, depth + 1, 0);
        }
        TNode &n = nodes_[size_t(id)];
        n.left = left; n.right = right; n.type = PT_BRANCH;
        // surrounding_box (src/bvh/aabb.h:41-55)
        const Box &a = nodes_[size_t(left)].box, &b = nodes_[size_t(right)].box;
        for(int k = 0; k < 3; k++) {
            n.box.lo[k] = a.lo[k] < b.lo[k] ? a.lo[k] : b.lo[k];
            n.box.hi[k] = a.hi[k] > b.hi[k] ? a.hi[k] : b.hi[k];
        }
        return id;
    }

    int32_t median(int32_t begin, int32_t end, const Box &cb) {
        int axis = 0;
        float ext = cb.hi[0] - cb.lo[0];
        for(int a = 1; a < 3; a++) if(cb.hi[a] - cb.lo[a] > ext) { ext = cb.hi[a] - cb.lo[a]; axis = a; }
        int32_t mid = begin + (end - begin)/2;
        std::nth_element(prims_.begin() + begin, prims_.begin() + mid, prims_.begin() + end,
                         [axis](const Prim &x, const Prim &y) {
                             return x.centroid[axis] < y.centroid[axis] ||
                                    (x.centroid[axis] == y.centroid[axis] && (x.type < y.type || (x.type == y.type && x.id < y.id)));
                         });
        return mid;
    }

    int32_t split(int32_t begin, int32_t end, const Box &cb, int depth) {
        int32_t n = end - begin;
        if(depth >= kMedianDepth || n <= 2) return median(begin, end, cb);
        double best = std::numeric_limits<double>::infinity();
        int best_axis = -1, best_bin = -1;
        for(int axis = 0; axis < 3; axis++) {
            float lo = cb.lo[axis], hi = cb.hi[axis];
            if(!(hi > lo)) continue;
            double scale = kBins / (double(hi) - lo);
            Box bins[kBins]; int counts[kBins] = {0};
            for(int b = 0; b < kBins; b++) bins[b].reset();
            for(int32_t i = begin; i < end; i++) {
                int b = int((prims_[size_t(i)].centroid[axis] - lo)*scale);
                b = b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
                counts[b]++;
                bins[b].grow(prims_[size_t(i)].box);
            }
            double right_area[kBins]; int right_count[kBins];
            Box acc; acc.reset(); int cnt = 0;
            for(int b = kBins - 1; b > 0; b--) {
                acc.grow(bins[b]); cnt += counts[b];
                right_area[b] = acc.area(); right_count[b] = cnt;
            }
            acc.reset(); cnt = 0;
            for(int b = 0; b < kBins - 1; b++) {
                acc.grow(bins[b]); cnt += counts[b];
                if(cnt == 0 || right_count[b + 1] == 0) continue;
                double cost = acc.area()*cnt + right_area[b + 1]*right_count[b + 1];
                if(cost < best) { best = cost; best_axis = axis; best_bin = b; }
            }
        }
        if(best_axis < 0) return median(begin, end, cb);
        float lo = cb.lo[best_axis], hi = cb.hi[best_axis];
        double scale = kBins / (double(hi) - lo);
        auto it = std::partition(prims_.begin() + begin, prims_.begin() + end, [&](const Prim &p) {
            int b = int((p.centroid[best_axis] - lo)*scale);
            b = b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
            return b <= best_bin;
        });
        int32_t mid = int32_t(it - prims_.begin());
        if(mid == begin || mid == end) return median(begin, end, cb);
        return mid;
    }
};

} // namespace

std::vector<BuildPrim> gather_prims(const FlatScene &scene) {
    std::vector<BuildPrim> prims;
    prims.reserve(scene.triangles.size() + scene.spheres.size());
    for(size_t i = 0; i < scene.triangles.size(); i++) {
        Box b = triangle_box(scene.triangles[i]);
        BuildPrim p{}; p.type = PT_TRIANGLE; p.id = int32_t(i);
        for(int a = 0; a < 3; a++) { p.lo[a] = b.lo[a]; p.hi[a] = b.hi[a]; }
        prims.push_back(p);
    }
    for(size_t i = 0; i < scene.spheres.size(); i++) {
        Box b = sphere_box(scene.spheres[i]);
        BuildPrim p{}; p.type = PT_SPHERE; p.id = int32_t(i);
        for(int a = 0; a < 3; a++) { p.lo[a] = b.lo[a]; p.hi[a] = b.hi[a]; }
        prims.push_back(p);
    }
    if(prims.size() >= size_t(INT32_MAX)/2) throw Error(PT_INVALID_ARGUMENT, "too many primitives for 32-bit node ids");
    return prims;
}

void export_preorder(FlatScene &scene, const std::vector<BuildNode> &nodes, int32_t root) {
    scene.nodes.clear();
    scene.max_depth = 0;
    if(root < 0) { scene.root = -1; return; }
    // preorder export, as flat_exporter::object emits nodes (src/flat/flat_export.h:100-114)
    scene.nodes.reserve(nodes.size());
    struct Item { int32_t temp; int depth; int32_t parent; int side; };
    std::vector<Item> stack{{root, 1, -1, 0}};
    while(!stack.empty()) {
        Item it = stack.back(); stack.pop_back();
        const BuildNode &t = nodes[size_t(it.temp)];
        int32_t id = int32_t(scene.nodes.size());
        pt_node n{};
        n.minimum = {t.lo[0], t.lo[1], t.lo[2]};
        n.maximum = {t.hi[0], t.hi[1], t.hi[2]};
        n.type = t.type; n.left = -1; n.right = -1; n.primitive = t.type == PT_BRANCH ? -1 : t.prim;
        scene.nodes.push_back(n);
        scene.max_depth = std::max(scene.max_depth, it.depth);
        if(scene.max_depth > kStackCapacity) throw Error(PT_INVALID_ARGUMENT, "BVH deeper than 64 levels");
        if(it.parent >= 0) {
            if(it.side == 0) scene.nodes[size_t(it.parent)].left = id;
            else scene.nodes[size_t(it.parent)].right = id;
        }
        if(t.type == PT_BRANCH) {
            stack.push_back({t.right, it.depth + 1, id, 1});
            stack.push_back({t.left, it.depth + 1, id, 0});
        }
    }
    scene.root = 0;
}

std::vector<BuildNode> sah_tree(const std::vector<BuildPrim> &gathered, int threads, int32_t &root) {
    std::vector<Prim> prims;
    prims.reserve(gathered.size());
    for(const BuildPrim &g : gathered) {
        Prim p;
        for(int a = 0; a < 3; a++) { p.box.lo[a] = g.lo[a]; p.box.hi[a] = g.hi[a]; p.centroid[a] = 0.5f*(g.lo[a] + g.hi[a]); }
        p.type = g.type; p.id = g.id;
        prims.push_back(p);
    }
    Builder builder(prims, threads < 1 ? hardware_threads() : threads);
    root = builder.run();
    std::vector<BuildNode> nodes(builder.nodes_.size());
    for(size_t i = 0; i < nodes.size(); i++) {
        const TNode &t = builder.nodes_[i];
        BuildNode &n = nodes[i];
        for(int a = 0; a < 3; a++) { n.lo[a] = t.box.lo[a]; n.hi[a] = t.box.hi[a]; }
        n.left = t.left; n.right = t.right; n.type = t.type; n.prim = t.prim;
    }
    return nodes;
}

void build_sah(FlatScene &scene, int threads) {
    int32_t root = -1;
    std::vector<BuildNode> nodes = sah_tree(gather_prims(scene), threads, root);
    export_preorder(scene, nodes, root);
}

} // namespace ptb
