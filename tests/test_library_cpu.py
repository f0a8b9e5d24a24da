"""CPU checks of the product library: C ABI exports, host validation, builders, generators.

No kernel runs here; pt_scene_create validates on the host before it looks for a device, so
rejections are testable without a GPU.
"""
from __future__ import annotations

import ctypes as C
import re
import sys
from pathlib import Path

import numpy as np
import pytest

import ptb200 as pt
from oracle_bind import Oracle, RefCpu, REF_CPU_SO, ORACLE_SO

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
G = np.load(Path(__file__).parent / "golden" / "reference_golden.npz")


def declared(header: Path) -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:pt_status|int|const char \*|void)\s+\*?(pt_\w+)\s*\(", text, flags=re.M)))


@pytest.mark.parametrize("header", sorted((ROOT / "include").glob("*.h")), ids=lambda p: p.name)
def test_library_exports_every_declared_symbol(header):
    lib = C.CDLL(str(pt.LIBRARY_PATH))
    names = declared(header)
    assert names, header
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_oracle_library_loads():
    assert ORACLE_SO.exists()
    lib = C.CDLL(str(ORACLE_SO))
    for n in ("or_trace_world", "or_query", "or_add_samples", "or_validate", "or_scene_lights"):
        assert hasattr(lib, n)


def golden_scene(prefix):
    return pt.FlatScene(G[f"{prefix}_triangles"], G[f"{prefix}_spheres"], G[f"{prefix}_nodes"],
                        G[f"{prefix}_materials"], G[f"{prefix}_textures"], G[f"{prefix}_pixels"],
                        int(G[f"{prefix}_root"]), int(G[f"{prefix}_max_depth"]))


def mutations(s: pt.FlatScene):
    """The rejections of tests/flat_tests.cpp:163-190 plus a few of validate_flat_scene's rules."""
    out = []
    m = s.copy(); m.nodes["left"][m.root] = 9999; out.append(("dangling child", m))
    m = s.copy(); m.nodes["left"][m.root] = m.root; out.append(("cycle", m))
    m = s.copy(); m.triangles["material_id"][0] = -1; out.append(("bad material", m))
    m = s.copy(); m.nodes["maximum"][m.root] = (-99, -99, -99); out.append(("inverted root box", m))
    m = s.copy(); m.max_depth += 1; out.append(("wrong depth", m))
    m = s.copy(); m.triangles["v0"][0] = (np.inf, 0, 0); out.append(("nonfinite vertex", m))
    m = s.copy(); m.materials["type"][0] = 7; out.append(("bad material type", m))
    m = s.copy(); m.spheres["radius"][0] = -1; out.append(("negative radius", m))
    m = s.copy(); m.triangles["smooth"][0] = 2; out.append(("smooth flag", m))
    return out


def test_validation_rejects_like_the_reference():
    lib = pt.library()
    oracle = Oracle()
    ref = RefCpu() if REF_CPU_SO.exists() else None
    base = golden_scene("cornell")
    for name, s in mutations(base):
        d = s.desc()
        h = C.c_void_p()
        st = lib.pt_scene_create(C.byref(d), C.byref(h))
        assert st == 2, (name, st)
        assert not oracle.validate(s), name
        if ref:
            assert not ref.validate(s), name
    assert oracle.validate(base)


def test_valid_scene_without_device_reports_no_device():
    ok, _ = pt.cuda_device_available()
    if ok:
        pytest.skip("a CUDA device is present")
    scene = golden_scene("cornell")   # keeps the arrays alive while the call reads them
    d = scene.desc()
    h = C.c_void_p()
    assert pt.library().pt_scene_create(C.byref(d), C.byref(h)) == 7


def test_cornell_workload():
    s, cam = pt.cornell_box(320, 200)
    assert len(s.triangles) == 20 and len(s.spheres) == 3
    oracle = Oracle()
    assert oracle.validate(s)
    lights, area = oracle.lights(s)
    assert len(lights) == 2 and abs(area - 0.13 * 0.11) < 1e-6
    emit = s.materials[s.triangles["material_id"]]["type"] == pt.LIGHT_MAT
    assert emit.sum() == 2
    assert np.isclose(s.materials["fuzz"], 0.1).any() and np.isclose(s.materials["ref_idx"], 1.5).any()


def test_sah_builder_output_is_valid_and_keeps_ids():
    s, _ = pt.procedural_scene(96, 60, sphere_count=3, segments=64, rings=33, seed=9, random_triangles=500)
    assert len(s.triangles) == 3 * 2 * 64 * 32 + 500 + 2 + 2
    oracle = Oracle()
    assert oracle.validate(s)
    if REF_CPU_SO.exists():
        assert RefCpu().validate(s)
    assert s.max_depth <= 64
    leaves = s.nodes[s.nodes["type"] == pt.TRIANGLE_TYPE]
    assert sorted(leaves["primitive"]) == list(range(len(s.triangles)))
    again = s.build_bvh(threads=1)
    assert oracle.validate(again)


def test_quantised_four_wide_tree_contains_every_child_box():
    """The walked four-wide nodes hold each child's box as 8-bit bounds on a power-of-two grid:
    the dequantised box must contain the float box it stands for (the box tests are conservative
    filters only then), and empty slots must be inverted.  Checked on the host for a displaced-
    sphere scene with a triangle soup, a scene with spheres and the Cornell box."""
    scenes = [pt.procedural_scene(96, 60, sphere_count=4, segments=64, rings=33, seed=5, random_triangles=3000,
                                  soup_edge_min=1e-3, soup_edge_max=1e-2)[0],
              pt.procedural_scene(96, 60, sphere_count=2, segments=16, rings=9, seed=2, box_size=1000.0,
                                  radius_min=1.0, radius_max=40.0)[0],
              pt.cornell_box(64, 40)[0]]
    for s in scenes:
        nodes, bad = pt.layout_check(s)
        assert nodes > 0 and bad == 0, (nodes, bad)


def test_quantised_tree_is_conservative_at_extreme_scales():
    """The quantised child bounds stay conservative far from the origin (coordinates near 1e5),
    for tiny geometry (a 1e-4 scale), and with a degenerate (zero-area) triangle in the scene."""
    base, _ = pt.procedural_scene(64, 40, sphere_count=3, segments=24, rings=13, seed=4, random_triangles=400)
    cases = []
    for scale, shift in ((1.0e1, 1.0e5), (1.0e-4, 0.0), (1.0, -3.0e3)):
        s = base.copy()
        for f in ("v0", "v1", "v2"):
            s.triangles[f] = s.triangles[f] * np.float32(scale) + np.float32(shift)
        s.spheres["center"] = s.spheres["center"] * np.float32(scale) + np.float32(shift)
        s.spheres["radius"] = s.spheres["radius"] * np.float32(scale)
        cases.append(s.build_bvh())
    s = base.copy()
    s.triangles["v1"][7] = s.triangles["v0"][7]
    s.triangles["v2"][7] = s.triangles["v0"][7]
    cases.append(s.build_bvh())
    for s in cases:
        nodes, bad = pt.layout_check(s)
        assert nodes > 0 and bad == 0, (nodes, bad)


def test_procedural_scene_counts():
    """The 1M-triangle scene: 16 spheres of 2*256*128 = 65,536 triangles, floor and light quads."""
    p = pt.procedural_params()
    assert (p.sphere_count, p.segments, p.rings) == (16, 256, 129)
    assert 2 * p.segments * (p.rings - 1) == 65536


def test_host_ray_generators_are_deterministic():
    s, cam = pt.cornell_box(64, 40)
    a = pt.camera_rays(cam, 64, 40, 5, 100, 512)
    b = pt.camera_rays(cam, 64, 40, 5, 100, 512)
    assert a.tobytes() == b.tobytes()
    c = pt.camera_rays(cam, 64, 40, 5, 0, 612)[100:]
    assert a.tobytes() == c.tobytes()
    r1, t1 = pt.surface_rays(s, 3, 0, 1000, shadow=True, threads=1)
    r2, t2 = pt.surface_rays(s, 3, 0, 1000, shadow=True, threads=8)
    assert r1.tobytes() == r2.tobytes() and t1.tobytes() == t2.tobytes()
    hits = Oracle().query(s, a)
    b1 = pt.bounce_rays(s, a, hits, 2, 0, threads=1)
    b2 = pt.bounce_rays(s, a, hits, 2, 0, threads=4)
    assert b1.tobytes() == b2.tobytes()
    n = np.linalg.norm(b1["direction"].astype(np.float64), axis=1)
    assert np.all(np.abs(n - 1) < 1e-5)


def test_oracle_lowest_id_tie_rule():
    """transport_tests' pruning scene (tests/transport_tests.cpp:54-78): the reference keeps the later
    coincident sphere and prunes the far branch (2 primitive tests vs 3 for brute force); the
    lowest-id rule keeps sphere 0."""
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
    tex = np.zeros(1, pt.TEXTURE)
    s = pt.FlatScene(None, spheres, nodes, mats, tex, None, 0, 3)
    ray = np.zeros(1, pt.RAY)
    ray[0] = ((0, 0, 3), (0, 0, -1), 0)
    o = Oracle()
    compat = o.query_compat(s, ray)
    assert compat["rec"]["material_id"][0] == 1 and compat["rec"]["t"][0] == 2.0
    h, st = o.query(s, ray, tie_lowest=False, stats=True)
    hb, stb = o.query(s, ray, tie_lowest=False, stats=True, brute=True)
    assert st["primitives"][0] == 2 and stb["primitives"][0] == 3
    low = o.query(s, ray, tie_lowest=True)
    assert low["primitive_id"][0] == 0
    # the tie counter sees both coincident spheres at t = 2 (one other primitive at that distance)
    hits, ties = o.query_ties(s, ray)
    assert hits.tobytes() == low.tobytes() and ties[0] == 1
    ray2 = ray.copy()
    ray2[0]["origin"] = (0.5, 0.5, -4)           # reaches only the far sphere: no tie
    assert o.query_ties(s, ray2)[1][0] == 0


def test_bench_samples_and_launch_counts():
    """bench.py's seeded random subsets and its count of kernels per query call."""
    import bench
    a = bench.random_indices(1 << 20, 1000, 7)
    assert len(a) == 1000 and len(np.unique(a)) == 1000 and (np.diff(a.astype(np.int64)) > 0).all()
    assert np.array_equal(a, bench.random_indices(1 << 20, 1000, 7)) and a.max() < (1 << 20)
    assert bench.walk_launches_per_query(True) == 8 and bench.walk_launches_per_query(False) == 1
    args = bench.parse([])
    assert args.steps >= 1 and args.warmup >= 3 and args.parity_rays == 1 << 20 and args.log2_rays == 25


def test_ray_records_are_the_reference_ray_layout(tmp_path):
    """Ray dumps (bench.py --dump-rays) are raw records of the reference's ray (src/core/ray.h:30-32:
    origin vec3, direction vec3, time float = 28 bytes); written and read back unchanged."""
    assert pt.RAY.itemsize == 28
    assert [pt.RAY.fields[k][1] for k in ("origin", "direction", "time")] == [0, 12, 24]
    s, cam = pt.cornell_box(32, 20)
    rays = pt.camera_rays(cam, 32, 20, 1, 0, 1000)
    f = tmp_path / "camera.ray"
    rays.view(np.uint8).tofile(f)
    assert f.stat().st_size == 28 * 1000
    assert np.fromfile(f, dtype=pt.RAY).tobytes() == rays.tobytes()
