"""Regenerates the golden fixtures in tests/golden/ from the reference's own code.

Run in a container that has the reference's sources (oracle/_ref/ built by `make -C oracle`):

    python tests/golden/make_golden.py

Every expected value below comes from the reference's functions compiled from its sources
(oracle/_ref/libref_cpu.so: trace_world, trace_pixel_sample, scene_lights, pixel_rng,
display_pixels, flatten_scene, obj_scene).  The committed .npz files let the CPU test suite pin
the oracle without the reference present.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "cuda-path-tracer_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

import ptb200 as pt  # noqa: E402
from oracle_bind import RefCpu  # noqa: E402

REF_ASSETS = Path(os.environ.get("PT_REFERENCE_DIR", "/root/reference")) / "assets" / "models"


def scene_arrays(prefix: str, s: pt.FlatScene) -> dict:
    return {f"{prefix}_triangles": s.triangles, f"{prefix}_spheres": s.spheres, f"{prefix}_nodes": s.nodes,
            f"{prefix}_materials": s.materials, f"{prefix}_textures": s.textures, f"{prefix}_pixels": s.pixels,
            f"{prefix}_root": np.int32(s.root), f"{prefix}_max_depth": np.int32(s.max_depth)}


def probe_rays(scene: pt.FlatScene, count: int, seed: int) -> np.ndarray:
    """Rays through the scene bounds in the three families of tests/mesh_validation.cpp:51-74
    (axis-parallel from outside, interior with non-unit directions, aimed at triangles), plus
    rays with zero and signed-zero direction components."""
    rng = np.random.default_rng(seed)
    lo = scene.nodes["minimum"][scene.root].astype(np.float64)
    hi = scene.nodes["maximum"][scene.root].astype(np.float64)
    center, extent = 0.5 * (lo + hi), hi - lo
    radius = float(np.linalg.norm(extent))
    rays = np.zeros(count, pt.RAY)
    for i in range(count):
        kind = i % 4
        if kind == 0:
            axis, sign = (i // 4) % 3, (1 if (i // 12) % 2 else -1)
            o = center + 1.4 * (rng.random(3) - 0.5) * extent
            o[axis] = center[axis] + sign * radius
            d = np.zeros(3)
            d[axis] = -sign
            if (i // 24) % 2:
                d[(axis + 1) % 3] = -0.0
        elif kind == 1:
            o = lo + rng.random(3) * extent
            d = rng.random(3) - 0.5
        elif kind == 2 and len(scene.triangles):
            t = scene.triangles[rng.integers(len(scene.triangles))]
            target = 0.23 * t["v0"] + 0.31 * t["v1"] + 0.46 * t["v2"]
            d = target - (center + radius * (rng.random(3) - 0.5))
            o = target - d
        else:
            o = center + (rng.random(3) - 0.5) * extent
            d = (rng.random(3) - 0.5) * (10.0 ** rng.integers(-6, 3))
        rays[i]["origin"], rays[i]["direction"], rays[i]["time"] = o, d, 0.5
    return rays


def main() -> None:
    ref = RefCpu()
    out = {}

    # PCG streams (src/renderer/random.h)
    pairs = [(0, 0), (1, 0), (1, 1), (7, 12345), (42, 54), (42, 55), (2**40 + 3, 2**33 + 1), (2**64 - 1, 640_000)]
    out["rng_pairs"] = np.array(pairs, np.uint64)
    us, raws = zip(*(ref.rng_draws(s, p, 64) for s, p in pairs))
    out["rng_uniform"], out["rng_raw"] = np.stack(us), np.stack(raws)

    # Cornell box: ray queries (BVH and brute) and a depth-50 progressive render
    cornell, cam = pt.cornell_box(32, 20)
    out.update(scene_arrays("cornell", cornell))
    out["cornell_camera"] = cam
    rays = np.concatenate([pt.camera_rays(cam, 32, 20, 1, 0, 1024), probe_rays(cornell, 1024, 5)])
    out["cornell_rays"] = rays
    for brute in (0, 1):
        res, st = ref.trace_world(cornell, rays, brute=bool(brute))
        out[f"cornell_result_brute{brute}"], out[f"cornell_stats_brute{brute}"] = res, st
    tmax = np.where(np.arange(len(rays)) % 2 == 0, np.float32(1.5), np.float32(3.4e38)).astype(np.float32)
    out["cornell_tmax"] = tmax
    out["cornell_result_tmax"], out["cornell_stats_tmax"] = ref.trace_world(cornell, rays, tmax=tmax)
    for mis in (1, 0):
        sums, rng, nrays = ref.render(cornell, cam, 32, 20, 1, [2, 1], mis=bool(mis))
        out[f"cornell_render_mis{mis}_sums"], out[f"cornell_render_mis{mis}_rng"] = sums, rng
        out[f"cornell_render_mis{mis}_rays"] = np.uint64(nrays)
    for debug in range(1, 6):
        sums, rng, nrays = ref.render(cornell, cam, 32, 20, 1, [2], debug=debug)
        out[f"cornell_debug{debug}_sums"], out[f"cornell_debug{debug}_rays"] = sums, np.uint64(nrays)

    # The reference's own scene pipeline on its sphere asset (obj_scene + flatten_scene)
    sphere, scam = ref.flat_obj(REF_ASSETS / "blender_sphere" / "sphere.obj", 19, 13, seed=7)
    out.update(scene_arrays("sphere", sphere))
    out["sphere_camera"] = scam
    srays = np.concatenate([pt.camera_rays(scam, 19, 13, 3, 0, 512), probe_rays(sphere, 512, 9)])
    out["sphere_rays"] = srays
    out["sphere_result"], out["sphere_stats"] = ref.trace_world(sphere, srays)
    sums, rng, nrays = ref.render(sphere, scam, 19, 13, 7, [3, 5])
    out["sphere_render_sums"], out["sphere_render_rng"], out["sphere_render_rays"] = sums, rng, np.uint64(nrays)
    img, prays = ref.portable_image(sphere, scam, 19, 13, 7, [3, 5])
    out["sphere_portable_image"], out["sphere_portable_rays"] = img, np.uint64(prays)

    # lighting_tests fixture (tests/lighting_tests.cpp:15-25), flattened by the reference
    for occluded in (0, 1):
        verts = [[[-10, -10, 0], [10, -10, 0], [0, 10, 0]], [[-0.2, -0.2, 2], [0.2, -0.2, 2], [0, 0.2, 2]]]
        colors, kinds = [[0.7, 0.7, 0.7], [10, 10, 10]], [0, 3]
        if occluded:
            verts.append([[-10, -10, 1], [10, -10, 1], [0, 10, 1]])
            colors.append([0, 0, 0])
            kinds.append(0)
        fixture = ref.flat_mesh(verts, colors, kinds, seed=7)
        out.update(scene_arrays(f"light{occluded}", fixture))
        fcam = ref.camera([0, 0, 0.1], [0, 0, 0], [0, 1, 0], 40, 19.0 / 13, 0, 0.1, 0, 1)
        out[f"light{occluded}_camera"] = fcam
        sums, rng, nrays = ref.render(fixture, fcam, 19, 13, 11, [16])
        out[f"light{occluded}_sums"], out[f"light{occluded}_rays"] = sums, np.uint64(nrays)

    # display_pixels (src/display/display_pixels.h:11-21)
    g = np.random.default_rng(3)
    lin = np.concatenate([g.random(300) * 1.2 - 0.1, [0, 1, 0.5, -0.0, np.nan, np.inf, 1e-9, 0.99999994, 2.0]]).astype(np.float32)
    lin = lin[: len(lin) // 3 * 3]
    out["pack_linear"], out["pack_rgba"] = lin, ref.display_pixels(lin)

    np.savez_compressed(HERE / "reference_golden.npz", **out)
    print("wrote", HERE / "reference_golden.npz", sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main()
