// pt_scene_host.cpp — validation, emitter table and BVH re-layout (host C++17).
#include <cfloat>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>
#include "pt_exact.h"
#include "pt_api_common.h"
#include "pt_host.h"

namespace ptb {

int hardware_threads() {
    unsigned n = std::thread::hardware_concurrency();
    return n ? int(n) : 1;
}

pt_scene_desc FlatScene::desc() const {
    pt_scene_desc d{};
    d.triangles = triangles.data(); d.triangle_count = triangles.size();
    d.spheres = spheres.data(); d.sphere_count = spheres.size();
    d.nodes = nodes.data(); d.node_count = nodes.size();
    d.materials = materials.data(); d.material_count = materials.size();
    d.textures = textures.data(); d.texture_count = textures.size();
    d.pixels = pixels.data(); d.pixel_bytes = pixels.size();
    d.root = root; d.max_depth = max_depth;
    return d;
}

namespace {
bool fin(const pt_vec3 &p) { return std::isfinite(p.x) && std::isfinite(p.y) && std::isfinite(p.z); }
float c(const pt_vec3 &p, int a) { return a == 0 ? p.x : (a == 1 ? p.y : p.z); }
bool valid(int32_t id, size_t count) { return id >= 0 && size_t(id) < count; }
void require(bool ok) { if(!ok) throw Error(PT_INVALID_SCENE, "invalid flat scene data"); }
} // namespace

// validate_flat_scene, src/flat/flat_validate.h:10-83
void validate_scene(const pt_scene_desc &s) {
    if((s.triangle_count && !s.triangles) || (s.sphere_count && !s.spheres) || (s.node_count && !s.nodes) ||
       (s.material_count && !s.materials) || (s.texture_count && !s.textures) || (s.pixel_bytes && !s.pixels))
        throw Error(PT_INVALID_ARGUMENT, "scene array pointer is null");
    for(size_t i = 0; i < s.texture_count; i++) {
        const pt_texture &t = s.textures[i];
        require(fin(t.color) && fin(t.scale) && fin(t.offset));
        require(t.type >= PT_TEX_CONSTANT && t.type <= PT_TEX_MAP);
        if(t.type == PT_TEX_IMAGE) {
            require(t.width > 0 && t.height > 0 && t.byte_offset >= 0);
            uint64_t end = uint64_t(t.byte_offset) + 3*uint64_t(t.width)*uint64_t(t.height);
            require(end <= s.pixel_bytes);
        } else if(t.type == PT_TEX_MAP) {
            require(valid(t.image_id, s.texture_count));
            require(s.textures[t.image_id].type == PT_TEX_IMAGE && (t.clamp == 0 || t.clamp == 1));
        }
    }
    for(size_t i = 0; i < s.material_count; i++) {
        const pt_material &m = s.materials[i];
        require(m.type >= PT_DIFFUSE && m.type <= PT_LIGHT && fin(m.albedo));
        require(std::isfinite(m.fuzz) && std::isfinite(m.ref_idx));
        if(m.type == PT_DIFFUSE || m.type == PT_LIGHT) require(valid(m.texture_id, s.texture_count));
        if(m.type == PT_GLASS) require(m.ref_idx > 0);
    }
    for(size_t i = 0; i < s.triangle_count; i++) {
        const pt_triangle &t = s.triangles[i];
        require(valid(t.material_id, s.material_count) && (t.smooth == 0 || t.smooth == 1));
        require(fin(t.v0) && fin(t.v1) && fin(t.v2) && fin(t.n0) && fin(t.n1) && fin(t.n2));
        require(fin(t.uv0) && fin(t.uv1) && fin(t.uv2));
    }
    for(size_t i = 0; i < s.sphere_count; i++) {
        const pt_sphere &p = s.spheres[i];
        require(valid(p.material_id, s.material_count) && fin(p.center) && std::isfinite(p.radius) && p.radius > 0);
    }
    if(s.root == -1) {
        require(s.node_count == 0 && s.triangle_count == 0 && s.sphere_count == 0 && s.max_depth == 0);
        return;
    }
    require(valid(s.root, s.node_count));
    if(s.node_count > size_t(INT32_MAX)) throw Error(PT_INVALID_SCENE, "invalid flat scene data");
    // Iterative post-order walk (the reference recurses; depth is bounded by 64 either way).
    std::vector<int> heights(s.node_count, 0);
    std::vector<unsigned char> active(s.node_count, 0);
    size_t visited = 0;
    struct Frame { int32_t id; int depth; int stage; int left_height; };
    std::vector<Frame> stack;
    int result = 0;
    auto enter = [&](int32_t id, int depth) -> int {   // returns height if already known, else 0 and pushes
        require(valid(id, s.node_count) && depth <= kStackCapacity && !active[id]);
        if(heights[id]) { require(depth + heights[id] - 1 <= kStackCapacity); return heights[id]; }
        active[id] = 1;
        visited++;
        const pt_node &n = s.nodes[id];
        require(fin(n.minimum) && fin(n.maximum));
        for(int a = 0; a < 3; a++) require(c(n.minimum, a) <= c(n.maximum, a));
        stack.push_back({id, depth, 0, 0});
        return 0;
    };
    int returned = enter(s.root, 1);
    if(returned) result = returned;
    while(!stack.empty()) {
        Frame &f = stack.back();
        const pt_node &n = s.nodes[f.id];
        int height = 1;
        if(n.type == PT_BRANCH) {
            if(f.stage == 0) {
                f.stage = 1;
                int h = enter(n.left, f.depth + 1);
                if(!h) continue;
                returned = h;
            }
            if(f.stage == 1) {
                f.left_height = returned;
                f.stage = 2;
                if(n.left != n.right) {
                    int h = enter(n.right, f.depth + 1);
                    if(!h) continue;
                    returned = h;
                } else returned = f.left_height;
            }
            int right_height = returned;
            height += std::max(f.left_height, right_height);
            for(int32_t child : {n.left, n.right}) {
                const pt_node &k = s.nodes[child];
                for(int a = 0; a < 3; a++) require(c(n.minimum, a) <= c(k.minimum, a) && c(n.maximum, a) >= c(k.maximum, a));
            }
        } else if(n.type == PT_TRIANGLE) {
            require(valid(n.primitive, s.triangle_count));
            const pt_triangle &t = s.triangles[n.primitive];
            for(const pt_vec3 &p : {t.v0, t.v1, t.v2})
                for(int a = 0; a < 3; a++) require(c(p, a) >= c(n.minimum, a) && c(p, a) <= c(n.maximum, a));
        } else if(n.type == PT_SPHERE) {
            require(valid(n.primitive, s.sphere_count));
            const pt_sphere &p = s.spheres[n.primitive];
            for(int a = 0; a < 3; a++)
                require(c(p.center, a) - p.radius >= c(n.minimum, a) && c(p.center, a) + p.radius <= c(n.maximum, a));
        } else require(false);
        active[f.id] = 0;
        heights[f.id] = height;
        returned = height;
        stack.pop_back();
        if(stack.empty()) result = height;
    }
    require(result == s.max_depth && visited == s.node_count);
}

// scene_lights, src/renderer/scene_view.h:10-28: cumulative emitter area in double.
std::vector<pt_light> scene_lights(const pt_scene_desc &s, float &total_area) {
    std::vector<pt_light> lights;
    double area = 0;
    auto add = [&](int type, int id, double size) {
        if(!(size > 0) || !std::isfinite(size)) return;
        area += size;
        if(!std::isfinite(area) || area > FLT_MAX) throw Error(PT_INVALID_ARGUMENT, "light area exceeds range");
        lights.push_back({type, id, float(area)});
    };
    for(size_t i = 0; i < s.triangle_count; i++) {
        const pt_triangle &t = s.triangles[i];
        if(s.materials[t.material_id].type == PT_LIGHT)
            add(PT_TRIANGLE, int(i), 0.5*(double)length(cross(mk(t.v1) - mk(t.v0), mk(t.v2) - mk(t.v0))));
    }
    for(size_t i = 0; i < s.sphere_count; i++) {
        const pt_sphere &p = s.spheres[i];
        if(s.materials[p.material_id].type == PT_LIGHT) add(PT_SPHERE, int(i), 4*M_PI*double(p.radius)*p.radius);
    }
    total_area = lights.empty() ? 0 : lights.back().cumulative_area;
    return lights;
}

namespace {
// Collapses the binary flat tree into four-wide nodes.  A child whose subtree holds at most
// kLeafMax primitives of one type becomes a leaf over its (consecutive, depth-first) slots;
// larger children are opened, largest surface area first, until a node has four children.
void build_wide(const pt_scene_desc &s, const std::vector<int32_t> &slot, int32_t tri_slots, HostLayout &out) {
    const pt_node *nodes = s.nodes;
    const size_t n = s.node_count;
    // subtree primitive count, type mask (1 triangle, 2 sphere) and first slot, post-order
    std::vector<int32_t> count(n, 0), first(n, INT32_MAX);
    std::vector<unsigned char> types(n, 0);
    std::vector<int32_t> order;
    order.reserve(n);
    std::vector<std::pair<int32_t, bool>> st{{s.root, false}};
    while(!st.empty()) {
        auto [id, expanded] = st.back(); st.pop_back();
        const pt_node &nd = nodes[id];
        if(nd.type != PT_BRANCH) {
            count[size_t(id)] = 1;
            types[size_t(id)] = nd.type == PT_TRIANGLE ? 1 : 2;
            first[size_t(id)] = nd.type == PT_TRIANGLE ? slot[size_t(id)] : tri_slots + slot[size_t(id)];
            continue;
        }
        if(expanded) {
            const int32_t a = nd.left, b = nd.right;
            count[size_t(id)] = count[size_t(a)] + (b != a ? count[size_t(b)] : 0);
            types[size_t(id)] = types[size_t(a)] | types[size_t(b)];
            first[size_t(id)] = std::min(first[size_t(a)], first[size_t(b)]);
            continue;
        }
        st.push_back({id, true});
        st.push_back({nd.left, false});
        if(nd.right != nd.left) st.push_back({nd.right, false});
    }
    auto leafable = [&](int32_t id) {
        return count[size_t(id)] <= kLeafMax && (types[size_t(id)] == 1 || types[size_t(id)] == 2);
    };
    auto area = [&](int32_t id) {
        const pt_node &nd = nodes[id];
        double dx = double(nd.maximum.x) - nd.minimum.x, dy = double(nd.maximum.y) - nd.minimum.y, dz = double(nd.maximum.z) - nd.minimum.z;
        return dx * dy + dy * dz + dz * dx;
    };
    const float inf = INFINITY;
    struct Work { int32_t flat; int32_t index; };
    std::vector<Work> work;
    auto make = [&](int32_t flat) {
        int32_t index = int32_t(out.nodes4.size());
        out.nodes4.push_back(Bvh4Node{});
        work.push_back({flat, index});
        return index;
    };
    // the root: a single leaf cluster becomes one child of a root node
    if(leafable(s.root)) {
        Bvh4Node r{};
        for(int k = 0; k < 4; k++) { r.lox[k] = r.loy[k] = r.loz[k] = inf; r.hix[k] = r.hiy[k] = r.hiz[k] = -inf; r.child[k] = kEmptyChild; }
        const pt_node &nd = nodes[s.root];
        r.lox[0] = nd.minimum.x; r.hix[0] = nd.maximum.x; r.loy[0] = nd.minimum.y; r.hiy[0] = nd.maximum.y;
        r.loz[0] = nd.minimum.z; r.hiz[0] = nd.maximum.z;
        r.child[0] = ~((first[size_t(s.root)] << 3) | (count[size_t(s.root)] - 1));
        out.nodes4.push_back(r);
        return;
    }
    if(size_t(tri_slots) + s.sphere_count >= (size_t(1) << 28)) { out.nodes4.clear(); return; }
    make(s.root);
    while(!work.empty()) {
        Work w = work.back(); work.pop_back();
        std::vector<int32_t> kids;
        const pt_node &nd = nodes[w.flat];
        kids.push_back(nd.left);
        if(nd.right != nd.left) kids.push_back(nd.right);
        while(kids.size() < 4) {
            int best = -1;
            double best_area = -1;
            for(size_t k = 0; k < kids.size(); k++) {
                const pt_node &c = nodes[kids[k]];
                if(c.type != PT_BRANCH || leafable(kids[k])) continue;
                double a = area(kids[k]);
                if(a > best_area) { best_area = a; best = int(k); }
            }
            if(best < 0) break;
            const pt_node &c = nodes[kids[size_t(best)]];
            kids[size_t(best)] = c.left;
            if(c.right != c.left) kids.insert(kids.begin() + best + 1, c.right);
        }
        Bvh4Node r{};
        for(int k = 0; k < 4; k++) { r.lox[k] = r.loy[k] = r.loz[k] = inf; r.hix[k] = r.hiy[k] = r.hiz[k] = -inf; r.child[k] = kEmptyChild; }
        for(size_t k = 0; k < kids.size(); k++) {
            const pt_node &c = nodes[kids[k]];
            r.lox[k] = c.minimum.x; r.hix[k] = c.maximum.x; r.loy[k] = c.minimum.y; r.hiy[k] = c.maximum.y;
            r.loz[k] = c.minimum.z; r.hiz[k] = c.maximum.z;
            if(leafable(kids[k])) r.child[k] = ~((first[size_t(kids[k])] << 3) | (count[size_t(kids[k])] - 1));
            else r.child[k] = make(kids[k]);
        }
        out.nodes4[size_t(w.index)] = r;
    }
}
} // namespace

Bvh4QNode quantize4(const Bvh4Node &n) {
    Bvh4QNode q{};
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const float *L[3] = {n.lox, n.loy, n.loz}, *H[3] = {n.hix, n.hiy, n.hiz};
    for(int k = 0; k < 4; k++) {
        q.child[k] = n.child[k];
        if(n.child[k] == kEmptyChild) continue;
        for(int a = 0; a < 3; a++) { lo[a] = std::min(lo[a], double(L[a][k])); hi[a] = std::max(hi[a], double(H[a][k])); }
    }
    float *P[3] = {&q.px, &q.py, &q.pz}, *S[3] = {&q.sx, &q.sy, &q.sz};
    for(int a = 0; a < 3; a++) {
        if(!(lo[a] <= hi[a])) { lo[a] = hi[a] = 0; }
        *P[a] = float(lo[a]);
        const double p = double(*P[a]), ext = hi[a] - p;
        int e = ext > 0 ? int(std::ceil(std::log2(ext / 255.0))) : -126;
        while(std::ldexp(255.0, e) < ext) e++;
        e = std::max(-126, std::min(127, e));
        const double step = std::ldexp(1.0, e);
        *S[a] = float(step);
        for(int k = 0; k < 4; k++) {
            uint32_t ql = 255, qh = 0;   // an empty slot: inverted
            if(n.child[k] != kEmptyChild) {
                ql = uint32_t(std::min(255.0, std::max(0.0, std::floor((double(L[a][k]) - p) / step))));
                qh = uint32_t(std::min(255.0, std::max(0.0, std::ceil((double(H[a][k]) - p) / step))));
            }
            q.qlo[a] |= ql << (8 * k);
            q.qhi[a] |= qh << (8 * k);
        }
    }
    return q;
}

// Re-layout: one 64-byte node per flat branch (reachable from the root), holding both
// children's boxes; leaves become slots into the 48-byte triangle / 32-byte sphere arrays,
// numbered in first-visit depth-first order so a subtree's leaves are contiguous.
HostLayout relayout(const pt_scene_desc &s) {
    HostLayout out;
    if(s.root < 0) { out.empty = 1; return out; }
    out.empty = 0;
    const pt_node *nodes = s.nodes;
    const pt_node &rootn = nodes[s.root];
    out.root_lo[0] = rootn.minimum.x; out.root_lo[1] = rootn.minimum.y; out.root_lo[2] = rootn.minimum.z;
    out.root_hi[0] = rootn.maximum.x; out.root_hi[1] = rootn.maximum.y; out.root_hi[2] = rootn.maximum.z;
    out.root_leaf = rootn.type != PT_BRANCH;
    std::vector<int32_t> inner(s.node_count, -1), slot(s.node_count, -1);
    std::vector<int32_t> tri_leaves, sphere_leaves;   // flat node ids per slot
    // Pass 1: number branches and leaves in preorder (left before right, as trace_world pops).
    std::vector<int32_t> stack{s.root};
    int32_t branches = 0;
    while(!stack.empty()) {
        int32_t id = stack.back(); stack.pop_back();
        const pt_node &n = nodes[id];
        if(n.type == PT_BRANCH) {
            if(inner[id] >= 0) continue;
            inner[id] = branches++;
            if(n.left != n.right) stack.push_back(n.right);
            stack.push_back(n.left);
        } else {
            if(slot[id] >= 0) continue;
            if(n.type == PT_TRIANGLE) { slot[id] = int32_t(tri_leaves.size()); tri_leaves.push_back(id); }
            else { slot[id] = int32_t(sphere_leaves.size()); sphere_leaves.push_back(id); }
        }
    }
    const int32_t tri_slots = int32_t(tri_leaves.size());
    auto leaf_ref = [&](int32_t id) -> int32_t {
        int32_t k = nodes[id].type == PT_TRIANGLE ? slot[id] : tri_slots + slot[id];
        return ~k;
    };
    auto child_ref = [&](int32_t id) { return nodes[id].type == PT_BRANCH ? inner[id] : leaf_ref(id); };
    const float inf = INFINITY;
    if(branches == 0) {
        // A root leaf: one node whose only child is that leaf.
        BvhNode n{};
        const pt_node &leaf = nodes[s.root];
        n.c0lox = leaf.minimum.x; n.c0hix = leaf.maximum.x; n.c0loy = leaf.minimum.y; n.c0hiy = leaf.maximum.y;
        n.c0loz = leaf.minimum.z; n.c0hiz = leaf.maximum.z;
        n.c1lox = inf; n.c1hix = -inf; n.c1loy = inf; n.c1hiy = -inf; n.c1loz = inf; n.c1hiz = -inf;
        n.child0 = leaf_ref(s.root); n.child1 = kEmptyChild;
        out.nodes.push_back(n);
    } else {
        out.nodes.resize(size_t(branches));
        for(size_t id = 0; id < s.node_count; id++) {
            if(inner[id] < 0) continue;
            const pt_node &p = nodes[id];
            BvhNode n{};
            const pt_node &a = nodes[p.left];
            n.c0lox = a.minimum.x; n.c0hix = a.maximum.x; n.c0loy = a.minimum.y; n.c0hiy = a.maximum.y;
            n.c0loz = a.minimum.z; n.c0hiz = a.maximum.z;
            n.child0 = child_ref(p.left);
            if(p.left != p.right) {
                const pt_node &b = nodes[p.right];
                n.c1lox = b.minimum.x; n.c1hix = b.maximum.x; n.c1loy = b.minimum.y; n.c1hiy = b.maximum.y;
                n.c1loz = b.minimum.z; n.c1hiz = b.maximum.z;
                n.child1 = child_ref(p.right);
            } else {
                n.c1lox = inf; n.c1hix = -inf; n.c1loy = inf; n.c1hiy = -inf; n.c1loz = inf; n.c1hiz = -inf;
                n.child1 = kEmptyChild;
            }
            out.nodes[size_t(inner[id])] = n;
        }
        // the root must be node 0: preorder numbering gives it index 0
    }
    out.tris.resize(tri_leaves.size());
    for(size_t k = 0; k < tri_leaves.size(); k++) {
        int32_t id = nodes[tri_leaves[k]].primitive;
        const pt_triangle &t = s.triangles[id];
        // The reference recomputes these per test (flat_intersect.h:10-13); same FP32 ops here.
        f3 e1 = mk(t.v1) - mk(t.v0), e2 = mk(t.v2) - mk(t.v0);
        float normal_length = length(cross(e1, e2));
        TriRecord r{};
        r.v0x = t.v0.x; r.v0y = t.v0.y; r.v0z = t.v0.z;
        r.eps = normal_length > 0 ? 0.0000001f * normal_length : INFINITY;   // !(normal_length > 0) never hits
        r.e1x = e1.x; r.e1y = e1.y; r.e1z = e1.z; r.id = id;
        r.e2x = e2.x; r.e2y = e2.y; r.e2z = e2.z; r.node = tri_leaves[k];
        out.tris[k] = r;
    }
    out.spheres.resize(sphere_leaves.size());
    for(size_t k = 0; k < sphere_leaves.size(); k++) {
        int32_t id = nodes[sphere_leaves[k]].primitive;
        const pt_sphere &p = s.spheres[id];
        SphereRecord r{};
        r.cx = p.center.x; r.cy = p.center.y; r.cz = p.center.z; r.radius = p.radius;
        r.id = id; r.node = sphere_leaves[k];
        out.spheres[k] = r;
    }
    // Four-wide collapse (trees only: a node reached twice keeps the two-wide layout).
    {
        std::vector<int32_t> parents(s.node_count, 0);
        bool shared = false;
        for(size_t id = 0; id < s.node_count && !shared; id++) {
            if(inner[id] < 0) continue;
            const pt_node &p = nodes[id];
            if(++parents[size_t(p.left)] > 1) shared = true;
            if(p.right != p.left && ++parents[size_t(p.right)] > 1) shared = true;
        }
        if(!shared) build_wide(s, slot, tri_slots, out);
    }
    for(const Bvh4Node &w : out.nodes4) out.nodes4q.push_back(quantize4(w));
    // brute order: leaves in flat node-array order
    for(size_t id = 0; id < s.node_count; id++) {
        if(nodes[id].type == PT_BRANCH || slot[id] < 0) continue;
        out.brute_order.push_back(~leaf_ref(int32_t(id)));
    }
    return out;
}

} // namespace ptb

extern "C" {

// Host-side check of the four-wide tree a scene would be walked with: rebuilds the re-layout as
// pt_scene_create does and, in exact (double) arithmetic, checks every child's dequantised bounds
// (origin + q * spacing) against the float bounds they stand for, and that empty slots are
// inverted on every axis.
pt_status pt_layout_check(const pt_scene_desc *desc, size_t *nodes, size_t *violations) {
    return ptb::guard([&]() {
        if(!desc || !nodes || !violations) throw ptb::Error(PT_INVALID_ARGUMENT, "null argument");
        ptb::validate_scene(*desc);
        const ptb::HostLayout layout = ptb::relayout(*desc);
        size_t bad = 0;
        for(size_t i = 0; i < layout.nodes4q.size(); i++) {
            const ptb::Bvh4Node &f = layout.nodes4[i];
            const ptb::Bvh4QNode &q = layout.nodes4q[i];
            const float *L[3] = {f.lox, f.loy, f.loz}, *H[3] = {f.hix, f.hiy, f.hiz};
            const double P[3] = {q.px, q.py, q.pz}, S[3] = {q.sx, q.sy, q.sz};
            for(int k = 0; k < 4; k++) {
                for(int a = 0; a < 3; a++) {
                    const uint32_t lo = (q.qlo[a] >> (8 * k)) & 0xffu, hi = (q.qhi[a] >> (8 * k)) & 0xffu;
                    if(q.child[k] != f.child[k]) { bad++; continue; }
                    if(f.child[k] == ptb::kEmptyChild) { bad += !(lo > hi); continue; }
                    bad += !(P[a] + lo * S[a] <= double(L[a][k]));
                    bad += !(P[a] + hi * S[a] >= double(H[a][k]));
                }
            }
        }
        *nodes = layout.nodes4q.size();
        *violations = bad;
    });
}

} // extern "C"
