"""OBJ/MTL import and the preview stage against the reference's own loader (no GPU).

tests/golden/obj_golden.npz holds what the reference's obj_scene + flatten_scene make of the
fixtures in tests/golden/obj/ (written by tests/golden/make_obj_golden.py).  The reference's tree
is a random-axis split and this library's is a binned SAH, so primitive and material ids differ;
the comparison resolves every triangle and sphere to its full record (positions, normals, UVs,
smooth flag, material with its texture chain and image bytes) and compares the sorted lists
bitwise, and the camera bitwise.
"""
from __future__ import annotations

import hashlib
from functools import lru_cache
from pathlib import Path

import numpy as np
import pytest

import ptb200 as pt

HERE = Path(__file__).parent / "golden"
G = np.load(HERE / "obj_golden.npz")
CASES = sorted({k.rsplit("_", 1)[0] for k in G.files if k.endswith("_args")})


def texture_key(textures, pixels, tid):
    if tid < 0:
        return ("none",)
    t = textures[tid]
    if t["type"] == pt.TEX_CONSTANT:
        return ("constant", t["color"].tobytes())
    if t["type"] == pt.TEX_IMAGE:
        n = int(t["width"]) * int(t["height"]) * 3
        off = int(t["byte_offset"])
        return ("image", int(t["width"]), int(t["height"]), hashlib.sha256(pixels[off:off + n].tobytes()).hexdigest())
    return ("map", t["color"].tobytes(), t["scale"].tobytes(), t["offset"].tobytes(), int(t["clamp"]),
            texture_key(textures, pixels, int(t["image_id"])))


def material_key(scene, mid):
    m = scene.materials[mid]
    kind = int(m["type"])
    if kind == pt.METAL:
        return ("metal", m["albedo"].tobytes(), float(m["fuzz"]))
    if kind == pt.GLASS:
        return ("glass", float(m["ref_idx"]))
    return (("diffuse", "light")[kind == pt.LIGHT_MAT], texture_key(scene.textures, scene.pixels, int(m["texture_id"])))


def triangle_keys(scene):
    keys = []
    mat = lru_cache(maxsize=None)(lambda mid: material_key(scene, mid))
    for t in scene.triangles:
        smooth = int(t["smooth"])
        normals = b"".join(t[f].tobytes() for f in ("n0", "n1", "n2")) if smooth else b""
        keys.append((b"".join(t[f].tobytes() for f in ("v0", "v1", "v2")), smooth, normals,
                     b"".join(t[f].tobytes() for f in ("uv0", "uv1", "uv2")), mat(int(t["material_id"]))))
    return sorted(keys, key=repr)


def sphere_keys(scene):
    return sorted(((s["center"].tobytes(), float(s["radius"]), material_key(scene, int(s["material_id"])))
                   for s in scene.spheres), key=repr)


def golden(name):
    tex = G[f"{name}_textures"]
    mats = G[f"{name}_materials"]
    s = pt.FlatScene(G[f"{name}_triangles"], G[f"{name}_spheres"], np.zeros(0, pt.NODE), mats, tex, G[f"{name}_pixels"], -1, 0)
    return s, G[f"{name}_camera"], G[f"{name}_args"]


@pytest.mark.parametrize("name", CASES)
def test_obj_scene_matches_reference_loader(name):
    want, want_cam, args = golden(name)
    w, h = int(args[0]), int(args[1])
    got, cam, warnings = pt.obj_scene(HERE / "obj" / "fixture.obj", w, h, args[2:5], args[5:8], args[8:11])
    assert cam.tobytes() == want_cam.tobytes()
    assert len(got.triangles) == len(want.triangles)
    assert triangle_keys(got) == triangle_keys(want)
    assert sphere_keys(got) == sphere_keys(want)
    assert "Skipped 2 degenerate triangles." in warnings          # the repeated-corner face and a collinear ear
    assert "simplified material mapping" in warnings and "missing_name" in warnings


def test_obj_scene_bvh_is_valid_and_complete():
    scene, _, _ = pt.obj_scene(HERE / "obj" / "fixture.obj", 64, 48)
    leaves = scene.nodes[scene.nodes["type"] != pt.BRANCH]
    assert sorted(leaves[leaves["type"] == pt.TRIANGLE_TYPE]["primitive"].tolist()) == list(range(len(scene.triangles)))
    assert sorted(leaves[leaves["type"] == pt.SPHERE_TYPE]["primitive"].tolist()) == [0, 1]


def test_obj_import_errors(tmp_path):
    with pytest.raises(ValueError, match="could not load OBJ"):
        pt.obj_scene(tmp_path / "none.obj", 10, 10)
    bad = tmp_path / "zero.obj"
    bad.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n")
    with pytest.raises(ValueError, match="zero value"):
        pt.obj_scene(bad, 10, 10)
    nomtl = tmp_path / "nomtl.obj"
    nomtl.write_text("mtllib absent.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    with pytest.raises(ValueError, match="could not load MTL"):
        pt.obj_scene(nomtl, 10, 10)
    empty = tmp_path / "empty.obj"
    empty.write_text("v 0 0 0\n")
    with pytest.raises(ValueError, match="no usable triangles"):
        pt.obj_scene(empty, 10, 10)
    jpg = tmp_path / "j.obj"
    (tmp_path / "j.mtl").write_text("newmtl j\nmap_Kd t.jpg\n")
    (tmp_path / "t.jpg").write_bytes(b"\xff\xd8\xff\xe0" + bytes(16))
    jpg.write_text("mtllib j.mtl\nusemtl j\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    with pytest.raises(ValueError, match="JPEG: bad marker length"):
        pt.obj_scene(jpg, 10, 10)
    from PIL import Image
    Image.fromarray(np.full((16, 16, 3), 90, np.uint8)).save(tmp_path / "t.jpg", progressive=True)
    with pytest.raises(ValueError, match="progressive"):
        pt.obj_scene(jpg, 10, 10)
    tri = tmp_path / "t.obj"
    tri.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    with pytest.raises(ValueError, match="nonzero scale"):
        pt.obj_scene(tri, 10, 10, scale=(1, 0, 1))
