"""Pins the CPU oracle (oracle/pt_oracle.c) to the reference.

Every expected value comes from tests/golden/reference_golden.npz, which
tests/golden/make_golden.py produced by running the reference's own code.  The comparisons
are bitwise: the oracle restates the reference's FP32/FP64 arithmetic operation for operation.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import ptb200 as pt
from oracle_bind import Oracle

G = np.load(Path(__file__).parent / "golden" / "reference_golden.npz")


def scene(prefix: str) -> pt.FlatScene:
    return pt.FlatScene(G[f"{prefix}_triangles"], G[f"{prefix}_spheres"], G[f"{prefix}_nodes"],
                        G[f"{prefix}_materials"], G[f"{prefix}_textures"], G[f"{prefix}_pixels"],
                        int(G[f"{prefix}_root"]), int(G[f"{prefix}_max_depth"]))


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


def same_bytes(a, b) -> bool:
    return a.dtype == b.dtype and a.shape == b.shape and a.tobytes() == b.tobytes()


def test_rng_streams(oracle):
    for (seed, pixel), expected in zip(G["rng_pairs"], G["rng_uniform"]):
        got = oracle.rng_draws(int(seed), int(pixel), expected.size)
        assert same_bytes(got, expected), (seed, pixel)


@pytest.mark.parametrize("brute", [0, 1])
def test_cornell_queries(oracle, brute):
    s = scene("cornell")
    got = oracle.query_compat(s, G["cornell_rays"], brute=bool(brute))
    assert same_bytes(got, G[f"cornell_result_brute{brute}"])
    hits, st = oracle.query(s, G["cornell_rays"], brute=bool(brute), tie_lowest=False, stats=True)
    ref_stats = G[f"cornell_stats_brute{brute}"]
    assert np.array_equal(st["boxes"], ref_stats["boxes"]) and np.array_equal(st["primitives"], ref_stats["primitives"])


def test_cornell_queries_with_tmax(oracle):
    s = scene("cornell")
    hits, st = oracle.query(s, G["cornell_rays"], tmax=G["cornell_tmax"], tie_lowest=False, stats=True)
    ref = G["cornell_result_tmax"]
    assert np.array_equal(hits["primitive_id"] >= 0, ref["hit"] == 1)
    m = ref["hit"] == 1
    assert np.array_equal(hits["t"][m].view(np.uint32), ref["rec"]["t"][m].view(np.uint32))
    assert np.array_equal(hits["primitive_id"][m], ref["rec"]["primitive_id"][m])
    assert np.array_equal(st["boxes"], G["cornell_stats_tmax"]["boxes"])


def test_reference_pipeline_scene_queries(oracle):
    s = scene("sphere")
    assert oracle.validate(s)
    got = oracle.query_compat(s, G["sphere_rays"])
    assert same_bytes(got, G["sphere_result"])


@pytest.mark.parametrize("mis", [1, 0])
def test_cornell_render_depth50(oracle, mis):
    s = scene("cornell")
    sums, rng, rays = oracle.render(s, G["cornell_camera"], 32, 20, 1, [2, 1], max_depth=50, mis=bool(mis))
    assert same_bytes(sums, G[f"cornell_render_mis{mis}_sums"])
    assert same_bytes(rng, G[f"cornell_render_mis{mis}_rng"])
    assert rays == int(G[f"cornell_render_mis{mis}_rays"])


@pytest.mark.parametrize("debug", range(1, 6))
def test_cornell_debug_views(oracle, debug):
    s = scene("cornell")
    sums, _, rays = oracle.render(s, G["cornell_camera"], 32, 20, 1, [2], max_depth=50, debug=debug)
    assert same_bytes(sums, G[f"cornell_debug{debug}_sums"])
    assert rays == int(G[f"cornell_debug{debug}_rays"])


def test_reference_pipeline_render(oracle):
    s = scene("sphere")
    sums, rng, rays = oracle.render(s, G["sphere_camera"], 19, 13, 7, [3, 5], max_depth=50)
    assert same_bytes(sums, G["sphere_render_sums"]) and same_bytes(rng, G["sphere_render_rng"])
    assert rays == int(G["sphere_render_rays"])
    # portable_renderer::image() divides through vec3::operator/= (reciprocal in double)
    assert same_bytes(oracle.image(sums, 8), G["sphere_portable_image"])
    assert rays == int(G["sphere_portable_rays"])


@pytest.mark.parametrize("occluded", [0, 1])
def test_lighting_fixture_render(oracle, occluded):
    s = scene(f"light{occluded}")
    sums, _, rays = oracle.render(s, G[f"light{occluded}_camera"], 19, 13, 11, [16], max_depth=50)
    assert same_bytes(sums, G[f"light{occluded}_sums"])
    assert rays == int(G[f"light{occluded}_rays"])


def test_display_pixels(oracle):
    lin = G["pack_linear"]
    got = oracle.pack_rgba(lin, 1, host_image=True)
    assert same_bytes(got, G["pack_rgba"])


def test_scene_lights(oracle):
    lights, area = oracle.lights(scene("cornell"))
    assert len(lights) == 2 and abs(area - 0.13 * 0.11) < 1e-6
