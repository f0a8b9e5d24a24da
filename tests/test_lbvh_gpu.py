"""The GPU linear-BVH builder (pt_flat_build_bvh_gpu): a valid flat tree whose answers equal
the SAH tree's.

Closest-hit queries resolve exact-distance ties to the lowest id, so their answers do not depend
on the tree: t, type and id are compared bitwise with the SAH tree's, and the any-hit occlusion
flags too.  The renderer keeps the reference's last-leaf tie rule, which does depend on the
tree, so its images are compared on a scene without coincident surfaces."""
from __future__ import annotations

import numpy as np
import pytest

import ptb200 as pt

pytestmark = pytest.mark.gpu


def check_tree(s: pt.FlatScene):
    nodes = s.nodes
    n_prims = len(s.triangles) + len(s.spheres)
    assert len(nodes) == 2 * n_prims - 1 and s.root == 0 and s.max_depth <= 64
    leaves = nodes[nodes["type"] != pt.BRANCH]
    assert sorted(leaves[leaves["type"] == pt.TRIANGLE_TYPE]["primitive"].tolist()) == list(range(len(s.triangles)))
    assert sorted(leaves[leaves["type"] == pt.SPHERE_TYPE]["primitive"].tolist()) == list(range(len(s.spheres)))
    branch = np.nonzero(nodes["type"] == pt.BRANCH)[0]
    lo = lambda k: nodes["minimum"][k]
    hi = lambda k: nodes["maximum"][k]
    L, R = nodes["left"][branch], nodes["right"][branch]
    assert (L > branch).all() and (R > branch).all()            # preorder
    # a branch's box is exactly the union of its children's
    assert np.array_equal(lo(branch), np.minimum(lo(L), lo(R))) and np.array_equal(hi(branch), np.maximum(hi(L), hi(R)))
    # leaf boxes are the SAH builder's (the reference's padded primitive boxes)
    sah = s.build_bvh()
    key = lambda t: np.lexsort((t["primitive"], t["type"]))
    a, b = leaves[key(leaves)], sah.nodes[sah.nodes["type"] != pt.BRANCH]
    b = b[key(b)]
    assert np.array_equal(a["minimum"], b["minimum"]) and np.array_equal(a["maximum"], b["maximum"])


@pytest.mark.parametrize("make", [lambda: pt.cornell_box(32, 20)[0],
                                  lambda: pt.procedural_scene(32, 20, sphere_count=4, segments=64, rings=33, seed=3)[0],
                                  lambda: pt.procedural_scene(32, 20, sphere_count=2, segments=32, rings=17, seed=5,
                                                              random_triangles=3000)[0]],
                         ids=["cornell", "spheres", "soup"])
def test_tree_is_valid(make):
    check_tree(make().build_bvh(gpu=True))


def test_small_scenes():
    s = pt.cornell_box(8, 8)[0]
    one = pt.FlatScene(s.triangles[:1], s.spheres[:0], s.nodes[:0], s.materials, s.textures, s.pixels, -1, 0)
    t = one.build_bvh(gpu=True)
    assert len(t.nodes) == 1 and t.root == 0 and t.nodes["type"][0] == pt.TRIANGLE_TYPE
    two = pt.FlatScene(s.triangles[:1], s.spheres[:1], s.nodes[:0], s.materials, s.textures, s.pixels, -1, 0)
    check_tree(two.build_bvh(gpu=True))


def test_queries_equal_the_sah_tree():
    flat, cam = pt.procedural_scene(160, 100, sphere_count=6, segments=96, rings=49, seed=11, random_triangles=20000)
    lb = flat.build_bvh(gpu=True)
    rays = pt.camera_rays(cam, 160, 100, 1, 0, 1 << 15)
    a, b = pt.Scene(flat), pt.Scene(lb)
    ha, hb = a.query(rays), b.query(rays)
    assert (ha["primitive_type"] != 0).mean() > 0.3
    assert ha.tobytes() == hb.tobytes()
    bounce = pt.bounce_rays(flat, rays, ha, 2, 0)
    assert a.query(bounce).tobytes() == b.query(bounce).tobytes()
    shadow, tmax = pt.surface_rays(flat, 3, 0, 1 << 14, shadow=True)
    oa = a.query(shadow, mode=pt.QUERY_ANY, tmax=tmax)["primitive_type"] != 0
    ob = b.query(shadow, mode=pt.QUERY_ANY, tmax=tmax)["primitive_type"] != 0
    assert np.array_equal(oa, ob) and 0.05 < oa.mean() < 0.95


def test_render_on_the_linear_bvh():
    flat, cam = pt.procedural_scene(64, 40, sphere_count=5, segments=64, rings=33, seed=2)
    a = pt.CudaRenderer(flat, cam, 64, 40, 1, max_depth=8)
    b = pt.CudaRenderer(flat.build_bvh(gpu=True), cam, 64, 40, 1, max_depth=8)
    a.add_samples(8)
    b.add_samples(8)
    same = (a.sums().reshape(-1, 3) == b.sums().reshape(-1, 3)).all(axis=1).mean()
    assert same > 0.999, same


def test_million_triangles():
    flat, _ = pt.procedural_scene(64, 40)
    lb = flat.build_bvh(gpu=True)
    assert len(lb.nodes) == 2 * (len(flat.triangles) + len(flat.spheres)) - 1 and lb.max_depth <= 64
