"""GPU parity of the closest-hit / any-hit kernels against the oracle and the reference.

Bar: the same hit primitive as the reference's traversal, exact-distance ties
resolved to the lowest (type, id), and t within 1e-6 relative.  The kernels reproduce the
reference's FP32 arithmetic, so these tests demand bit equality of t, which is stricter.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import ptb200 as pt
from oracle_bind import Oracle, RefCpu, RefGpu, REF_CPU_SO, REF_GPU_SO

pytestmark = pytest.mark.gpu
G = np.load(Path(__file__).parent / "golden" / "reference_golden.npz")
T_REL = 1e-6   # tolerance on t (the checks below are bitwise, which implies it)


def golden_scene(prefix):
    return pt.FlatScene(G[f"{prefix}_triangles"], G[f"{prefix}_spheres"], G[f"{prefix}_nodes"],
                        G[f"{prefix}_materials"], G[f"{prefix}_textures"], G[f"{prefix}_pixels"],
                        int(G[f"{prefix}_root"]), int(G[f"{prefix}_max_depth"]))


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


@pytest.fixture(params=[(1, 1), (1, 0), (0, 1)], ids=["wide-phased", "wide-loop", "binary"])
def layout(request):
    """Runs a test with each traversal form: four-wide nodes walked in node/leaf phases or in one
    loop, and the two-wide re-layout of the caller's tree."""
    wide, spec = request.param
    pt.query_layout(wide)
    pt.query_walk(spec)
    yield request.param
    pt.query_layout(1)
    pt.query_walk(1)


def assert_hits_equal(got, want):
    assert got.dtype == pt.HIT and want.dtype == pt.HIT
    assert np.array_equal(got["primitive_type"], want["primitive_type"])
    assert np.array_equal(got["primitive_id"], want["primitive_id"])
    m = want["primitive_type"] != 0
    assert np.array_equal(got["t"][m].view(np.uint32), want["t"][m].view(np.uint32))
    rel = np.abs(got["t"][m] - want["t"][m]) / np.maximum(np.abs(want["t"][m]), 1e-30)
    assert (rel <= T_REL).all()
    assert not got["error"].any()


def assert_trace_results(got, want):
    """Bitwise on every field, except the sphere UVs: those come from atan2f/asinf
    (get_sphere_uv, src/geometry/sphere_uv.h:7-13), whose CUDA and glibc results differ by a few
    ULP; the reference's own GPU build shows the same difference against its CPU build."""
    assert np.array_equal(got["hit"], want["hit"]) and np.array_equal(got["error"], want["error"])
    g, w = got["rec"], want["rec"]
    for f in ("t", "p", "normal", "material_id", "primitive_type", "primitive_id"):
        assert g[f].tobytes() == w[f].tobytes(), f
    sph = w["primitive_type"] == pt.SPHERE_TYPE
    for f in ("u", "v"):
        assert g[f][~sph].tobytes() == w[f][~sph].tobytes(), f
        assert np.allclose(g[f][sph], w[f][sph], rtol=0, atol=1e-6), f


@pytest.mark.parametrize("brute", [False, True])
def test_compat_matches_reference_golden(brute, layout):
    """cuda_query_rays semantics: full 56-byte trace_result, reference tie rule."""
    s = golden_scene("cornell")
    got = pt.cuda_query_rays(s, G["cornell_rays"], brute=brute)
    assert_trace_results(got, G[f"cornell_result_brute{int(brute)}"])


def test_compat_reference_pipeline_scene(layout):
    s = golden_scene("sphere")
    got = pt.cuda_query_rays(s, G["sphere_rays"])
    assert_trace_results(got, G["sphere_result"])


@pytest.mark.parametrize("prefix", ["cornell", "sphere", "light0", "light1"])
def test_closest_and_any_vs_oracle(oracle, prefix, layout):
    s = golden_scene(prefix)
    rays = G["cornell_rays"] if prefix == "cornell" else G["sphere_rays"] if prefix == "sphere" else \
        pt.camera_rays(G[f"{prefix}_camera"], 19, 13, 5, 0, 2048)
    dev = pt.Scene(s)
    assert_hits_equal(dev.query(rays), oracle.query(s, rays))
    got_any = dev.query(rays, mode=pt.QUERY_ANY)
    want_any = oracle.query(s, rays, mode=pt.QUERY_ANY)
    assert np.array_equal(got_any["primitive_type"] != 0, want_any["primitive_id"] >= 0)


def test_tmax_and_stats(oracle, layout):
    s = golden_scene("cornell")
    rays, tmax = G["cornell_rays"], G["cornell_tmax"]
    dev = pt.Scene(s)
    hits, stats = dev.query(rays, tmax=tmax, stats=True)
    assert_hits_equal(hits, oracle.query(s, rays, tmax=tmax))
    assert (stats["primitives"] >= (hits["primitive_type"] != 0)).all()


def test_exact_tie_lowest_id(layout):
    """transport_tests' pruning scene (tests/transport_tests.cpp:54-78): two coincident spheres.
    The reference keeps the later leaf (material 1); the query API's rule keeps the lowest id."""
    spheres = np.zeros(3, pt.SPHERE)
    spheres[0] = ((0, 0, 0), 1, 0)
    spheres[1] = ((0, 0, 0), 1, 1)
    spheres[2] = ((0, 0, -8), 1, 0)
    nodes = np.zeros(6, pt.NODE)
    nodes[0] = ((-1, -1, -9), (1, 1, 1), 0, 1, 4, -1)
    nodes[1] = ((-1, -1, -1), (1, 1, 1), 0, 2, 3, -1)
    nodes[2] = ((-1, -1, -1), (1, 1, 1), 2, -1, -1, 0)
    nodes[3] = ((-1, -1, -1), (1, 1, 1), 2, -1, -1, 1)
    nodes[4] = ((-1, -1, -9), (1, 1, -7), 0, 5, 5, -1)
    nodes[5] = ((-1, -1, -9), (1, 1, -7), 2, -1, -1, 2)
    mats = np.zeros(2, pt.MATERIAL)
    mats["type"], mats["texture_id"] = 0, 0
    tex = np.zeros(1, pt.TEXTURE)
    s = pt.FlatScene(None, spheres, nodes, mats, tex, None, 0, 3)
    ray = np.zeros(1, pt.RAY)
    ray[0] = ((0, 0, 3), (0, 0, -1), 0)
    compat = pt.cuda_query_rays(s, ray)
    assert compat["hit"][0] == 1 and compat["rec"]["material_id"][0] == 1 and compat["rec"]["t"][0] == 2.0
    hits = pt.Scene(s).query(ray)
    assert hits["primitive_id"][0] == 0 and hits["primitive_type"][0] == pt.SPHERE_TYPE and hits["t"][0] == 2.0


def test_empty_and_single_primitive_scenes(oracle, layout):
    empty = pt.FlatScene()
    rays = G["cornell_rays"][:64]
    hits = pt.Scene(empty).query(rays)
    assert (hits["primitive_type"] == 0).all() and (hits["primitive_id"] == -1).all()
    tri = np.zeros(1, pt.TRIANGLE)
    tri[0]["v0"], tri[0]["v1"], tri[0]["v2"] = (0, 0, 0), (1, 0, 0), (0, 1, 0)
    tri[0]["uv1"], tri[0]["uv2"] = (1, 0, 0), (0, 1, 0)
    mats = np.zeros(1, pt.MATERIAL)
    tex = np.zeros(1, pt.TEXTURE)
    one = pt.FlatScene(tri, None, None, mats, tex).build_bvh()
    assert one.root == 0 and len(one.nodes) == 1
    r = np.zeros(3, pt.RAY)
    r[0] = ((0.25, 0.25, 2), (0, 0, -2), 0.4)     # triangle_tests' front hit: t = 1
    r[1] = ((0.8, 0.8, 1), (0, 0, -1), 0)         # outside
    r[2] = ((0.5, 0.5, 1), (0, 0, -1), 0)         # on the hypotenuse edge: included
    got = pt.Scene(one).query(r, tmin=0.0)
    assert got["t"][0] == 1.0 and got["primitive_id"][0] == 0 and got["primitive_id"][1] == -1 and got["primitive_id"][2] == 0
    assert_hits_equal(got, oracle.query(one, r, tmin=0.0))


def test_brute_device_equals_bvh(oracle, layout):
    s, cam = pt.cornell_box(64, 40)
    dev = pt.Scene(s)
    torch = pytest.importorskip("torch")
    rays = pt.camera_rays(cam, 64, 40, 9, 0, 8192)
    d_rays = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
    a = torch.zeros(len(rays) * 16, dtype=torch.uint8, device="cuda")
    b = torch.zeros_like(a)
    dev.query_device(d_rays, len(rays), a)
    dev.query_device(d_rays, len(rays), b, brute=True)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_procedural_scene_vs_oracle(oracle, layout):
    """A 4-sphere, 64k-triangle displaced-sphere scene: camera rays and bounce rays."""
    torch = pytest.importorskip("torch")
    s, cam = pt.procedural_scene(96, 60, sphere_count=4, segments=128, rings=65, seed=3)
    dev = pt.Scene(s)
    n = 1 << 15
    prim = torch.zeros(n * 28, dtype=torch.uint8, device="cuda")
    pt.camera_rays_device(cam, 96, 60, 1, 0, n, prim)
    hits = torch.zeros(n * 16, dtype=torch.uint8, device="cuda")
    dev.query_device(prim, n, hits)
    bounce = torch.zeros_like(prim)
    dev.bounce_rays_device(prim, hits, n, 2, 0, bounce)
    hits2 = torch.zeros_like(hits)
    dev.query_device(bounce, n, hits2)
    torch.cuda.synchronize()
    host_prim = prim.cpu().numpy().view(pt.RAY)
    assert host_prim.tobytes() == pt.camera_rays(cam, 96, 60, 1, 0, n).tobytes()
    assert_hits_equal(hits.cpu().numpy().view(pt.HIT), oracle.query(s, host_prim))
    b = bounce.cpu().numpy().view(pt.RAY)
    assert_hits_equal(hits2.cpu().numpy().view(pt.HIT), oracle.query(s, b))
    # any-hit shadow rays between surface points
    sr, tmax = pt.surface_rays(s, 5, 0, 8192, shadow=True)
    got = dev.query(sr, mode=pt.QUERY_ANY, tmax=tmax)
    want = oracle.query(s, sr, mode=pt.QUERY_ANY, tmax=tmax)
    assert np.array_equal(got["primitive_type"] != 0, want["primitive_id"] >= 0)


def test_ray_order_keeps_answers(oracle, layout):
    """Batches of at least 2^18 rays are walked in (octant, origin Morton code) order: the hits
    and any-hit answers are the same bytes as walking the rays as given, and a sample of them
    equals the oracle's.  (The per-ray walk counters are not compared: in the phased walk a lane
    holding a leaf walks on while its warp finishes the node phase, so its counts depend on which
    rays share the warp.)"""
    torch = pytest.importorskip("torch")
    s, cam = pt.procedural_scene(160, 100, sphere_count=5, segments=96, rings=49, seed=8, random_triangles=5000)
    dev = pt.Scene(s)
    n = 1 << 18
    rays = torch.zeros(2 * n * 28, dtype=torch.uint8, device="cuda")
    hits = torch.zeros(n * 16, dtype=torch.uint8, device="cuda")
    pt.camera_rays_device(cam, 160, 100, 1, 0, n, rays)
    dev.query_device(rays, n, hits)
    dev.bounce_rays_device(rays, hits, n, 2, 0, rays[n * 28:])
    tmax = torch.rand(2 * n, generator=torch.Generator(device="cuda").manual_seed(3), device="cuda") * 20
    out = {}
    try:
        for order in (0, 1):
            pt.query_order(order)
            h = torch.zeros(2 * n * 16, dtype=torch.uint8, device="cuda")
            st = torch.zeros(2 * n * 8, dtype=torch.uint8, device="cuda")
            a = torch.zeros(2 * n * 16, dtype=torch.uint8, device="cuda")
            dev.query_device(rays, 2 * n, h, stats=st)
            dev.query_device(rays, 2 * n, a, mode=pt.QUERY_ANY, tmax=tmax)
            torch.cuda.synchronize()
            out[order] = (h.cpu().numpy(), a.cpu().numpy())
    finally:
        pt.query_order(2)
    for x, y in zip(out[0], out[1]):
        assert x.tobytes() == y.tobytes()
    got = out[1][0].view(pt.HIT)
    assert (got["primitive_type"] != 0).mean() > 0.3
    host = rays.cpu().numpy().view(pt.RAY)
    pick = np.r_[0:2048, n:n + 2048]
    assert_hits_equal(got[pick], oracle.query(s, host[pick]))


def test_ray_order_modes():
    """pt_query_order: 0 never orders, 1 orders batches of at least 2^18 rays, 2 (the default) only
    on scenes whose walked arrays exceed the L2 (a small scene: not ordered); other modes are
    rejected and leave the setting as it was."""
    s, _ = pt.procedural_scene(64, 64, sphere_count=2, segments=32, rings=17, seed=3)
    dev = pt.Scene(s)
    try:
        assert not dev.query_ordered(1 << 20)                # default mode 2, scene far below the L2
        pt.query_order(1)
        assert dev.query_ordered(1 << 18) and not dev.query_ordered((1 << 18) - 1)
        with pytest.raises(pt.PtError) as e:
            pt.query_order(3)
        assert e.value.status == 1                           # PT_INVALID_ARGUMENT
        assert dev.query_ordered(1 << 18)                    # still mode 1
        pt.query_order(0)
        assert not dev.query_ordered(1 << 20)
    finally:
        pt.query_order(2)


def _sample_rows(dev_u8, idx, width, dtype):
    import torch
    return dev_u8.view(-1, width)[torch.from_numpy(idx.astype(np.int64)).cuda()].cpu().numpy().view(dtype).reshape(-1)


@pytest.mark.skipif(not REF_CPU_SO.exists(), reason="reference CPU build absent")
def test_headline_scene_random_rays_vs_oracle_and_reference(oracle):
    """The benchmark's own scene (1,048,580 triangles) and ray generators at full size: 2^24
    camera rays and their 2^24 bounce rays walked in one 2^25-ray batch (key-ordered walk), and a
    seeded random 2^18 of them compared with the oracle (type, id, t bitwise, lowest-id ties) and
    with the reference's own trace_world wherever no exact-distance tie decides."""
    torch = pytest.importorskip("torch")
    s, cam = pt.procedural_scene(960, 600)
    dev = pt.Scene(s)
    half = 1 << 24
    rays = torch.empty(2 * half * 28, dtype=torch.uint8, device="cuda")
    hits = torch.empty(2 * half * 16, dtype=torch.uint8, device="cuda")
    pt.camera_rays_device(cam, 960, 600, 1, 0, half, rays)
    dev.query_device(rays, half, hits)
    dev.bounce_rays_device(rays, hits, half, 2, 0, rays[half * 28:])
    dev.query_device(rays, 2 * half, hits)
    torch.cuda.synchronize()
    idx = np.sort(np.random.default_rng(17).choice(2 * half, 1 << 18, replace=False))
    r = _sample_rows(rays, idx, 28, pt.RAY)
    got = _sample_rows(hits, idx, 16, pt.HIT)
    del rays, hits
    want, ties = oracle.query_ties(s, r)
    assert_hits_equal(got, want)
    res, _ = RefCpu().trace_world(s, r)
    hit = res["hit"] == 1
    assert np.array_equal(hit, got["primitive_type"] != 0)
    no_tie = hit & (ties == 0)
    assert np.array_equal(res["rec"]["primitive_id"][no_tie], got["primitive_id"][no_tie])
    assert np.array_equal(res["rec"]["t"][hit].view(np.uint32), got["t"][hit].view(np.uint32))
    assert (idx >= half).any() and (idx < half).any() and hit.mean() > 0.4


@pytest.mark.skipif(not REF_CPU_SO.exists(), reason="reference CPU build absent")
def test_microbenchmark_scene_closest_and_any_hit(oracle):
    """The traversal microbenchmark's scene kind at reduced size (16 displaced spheres of 16,384
    triangles and 65,536 random small triangles in a unit cube): camera rays and cosine surface
    rays (closest hit) and shadow rays between surface points (any hit), generated on the device,
    against the oracle and the reference's trace_world."""
    torch = pytest.importorskip("torch")
    s, cam = pt.procedural_scene(512, 512, sphere_count=16, segments=128, rings=65, box_size=1.0, radius_min=0.03,
                                 radius_max=0.08, floor=0, light_fraction=0.0, random_triangles=1 << 16, seed=3)
    dev = pt.Scene(s)
    n = 1 << 18
    rays = torch.empty(n * 28, dtype=torch.uint8, device="cuda")
    pt.camera_rays_device(cam, 512, 512, 3, 0, n // 2, rays)
    dev.surface_rays_device(4, 0, n // 2, rays[n // 2 * 28:])
    hits = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    dev.query_device(rays, n, hits)
    host = rays.cpu().numpy().view(pt.RAY)
    assert host[n // 2:].tobytes() == pt.surface_rays(s, 4, 0, n // 2).tobytes()
    got = hits.cpu().numpy().view(pt.HIT)
    pick = np.sort(np.random.default_rng(5).choice(n, 1 << 14, replace=False))
    want, ties = oracle.query_ties(s, host[pick])
    assert_hits_equal(got[pick], want)
    tmax = torch.empty(n * 4, dtype=torch.uint8, device="cuda")
    dev.surface_rays_device(5, 0, n, rays, tmax=tmax)
    dev.query_device(rays, n, hits, mode=pt.QUERY_ANY, tmax=tmax)
    host = rays.cpu().numpy().view(pt.RAY)
    tm = tmax.cpu().numpy().view(np.float32)
    sr, stm = pt.surface_rays(s, 5, 0, n, shadow=True)
    assert host.tobytes() == sr.tobytes() and tm.tobytes() == stm.tobytes()
    got = hits.cpu().numpy().view(pt.HIT)
    want = oracle.query(s, host[pick], mode=pt.QUERY_ANY, tmax=tm[pick])
    assert np.array_equal(got["primitive_type"][pick] != 0, want["primitive_id"] >= 0)
    res, _ = RefCpu().trace_world(s, host[pick], tmax=tm[pick])
    assert np.array_equal(got["primitive_type"][pick] != 0, res["hit"] == 1)
    assert 0.05 < (got["primitive_type"] != 0).mean() < 0.95


@pytest.mark.skipif(not REF_GPU_SO.exists(), reason="reference CUDA build absent")
def test_matches_reference_gpu_query(layout):
    """Our compatibility query and the reference's own cuda_query_rays on the same B200."""
    s = golden_scene("cornell")
    want = RefGpu().query(s, G["cornell_rays"])
    got = pt.cuda_query_rays(s, G["cornell_rays"])
    assert got.tobytes() == want.tobytes()


def test_invalid_scene_is_rejected():
    s = golden_scene("cornell").copy()
    s.nodes["left"][s.root] = 9999
    with pytest.raises(pt.PtError) as e:
        pt.Scene(s)
    assert e.value.status == 2


def deepest_chain_scene(levels: int = 64):
    """A tree of the greatest depth the reference's validator accepts (64 levels): every branch has
    a branch on the left and one triangle leaf on the right, 64 stacked triangles, the nearest
    (from below) at the bottom, so a ray along +z walks the whole chain."""
    tris = np.zeros(levels, pt.TRIANGLE)
    for k in range(levels):
        z = 0.05 * k
        tris[k]["v0"], tris[k]["v1"], tris[k]["v2"] = (-1, -1, z), (3, -1, z), (-1, 3, z)
        tris[k]["n0"] = tris[k]["n1"] = tris[k]["n2"] = (0, 0, 1)
    nodes = []

    def box(ids):
        lo = np.min([np.minimum(np.minimum(tris[i]["v0"], tris[i]["v1"]), tris[i]["v2"]) for i in ids], axis=0) - 1e-3
        hi = np.max([np.maximum(np.maximum(tris[i]["v0"], tris[i]["v1"]), tris[i]["v2"]) for i in ids], axis=0) + 1e-3
        return lo, hi

    def build(level, ids):           # ids: triangles of this subtree, nearest first
        me = len(nodes)
        nodes.append(None)
        lo, hi = box(ids)
        if level == levels:
            nodes[me] = (lo, hi, 1, -1, -1, ids[0])
            return me
        left = build(level + 1, ids[:-1])
        right = len(nodes)
        rlo, rhi = box(ids[-1:])
        nodes.append((rlo, rhi, 1, -1, -1, ids[-1]))
        nodes[me] = (lo, hi, 0, left, right, -1)
        return me
    build(1, list(range(levels)))
    arr = np.zeros(len(nodes), pt.NODE)
    for i, (lo, hi, t, l, r, p) in enumerate(nodes):
        arr[i] = (lo, hi, t, l, r, p)
    mats = np.zeros(1, pt.MATERIAL)
    mats[0]["albedo"] = (0.5, 0.5, 0.5)
    mats[0]["ref_idx"] = 1.0
    tex = np.zeros(1, pt.TEXTURE)
    tex[0]["color"] = (0.5, 0.5, 0.5)
    return pt.FlatScene(tris, np.zeros(0, pt.SPHERE), arr, mats, tex, np.zeros(0, np.uint8), 0, levels)


def test_deepest_valid_tree_matches_oracle_without_overflow(oracle, layout):
    """trace_world's stack holds 64 entries and the validator bounds the depth at 64, which keeps
    a validated tree from overflowing it (each level leaves at most one entry behind).  On the
    deepest chain the reference accepts, the oracle reports no overflow (error 0), and every
    traversal form gives the oracle's answers and error flags: closest hits from below and from
    above, and any-hit shadow rays."""
    s = deepest_chain_scene()
    dev = pt.Scene(s)
    g = np.random.default_rng(9)
    n = 4096
    rays = np.zeros(n, pt.RAY)
    xy = g.uniform(-0.9, 0.9, (n, 2))
    up = np.arange(n) % 2 == 0
    rays["origin"] = np.c_[xy, np.where(up, -1.0, 4.0)]
    rays["direction"] = np.c_[g.uniform(-0.05, 0.05, (n, 2)), np.where(up, 1.0, -1.0)]
    want = oracle.query(s, rays)
    assert not want["error"].any() and (want["primitive_type"] == 1).all()
    assert_hits_equal(dev.query(rays), want)
    assert set(np.unique(want["primitive_id"])) == {0, 63}
    tmax = np.full(n, 1.5, np.float32)
    got = dev.query(rays, mode=pt.QUERY_ANY, tmax=tmax)
    want_any = oracle.query(s, rays, mode=pt.QUERY_ANY, tmax=tmax)
    assert np.array_equal(got["primitive_type"] != 0, want_any["primitive_id"] >= 0)
    assert not got["error"].any()
