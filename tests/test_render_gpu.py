"""GPU parity of the wavefront renderer against the oracle and the reference's own renderer.

Bars: against the reference's CUDA renderer on the same B200 (same arithmetic, same CUDA math
functions) the linear sums, PCG states and ray counts are bit-identical; against the CPU oracle
(glibc transcendentals differ from CUDA's by a few ULP) the image's relative L2 error is below
1e-4 with equal ray counts, the bar the reference sets for its own GPU renderer
(tests/lighting_tests.cpp:86-92).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import ptb200 as pt
from oracle_bind import Oracle, RefGpu, REF_GPU_SO

pytestmark = pytest.mark.gpu
G = np.load(Path(__file__).parent / "golden" / "reference_golden.npz")
REL_L2 = 1e-4


def golden_scene(prefix):
    return pt.FlatScene(G[f"{prefix}_triangles"], G[f"{prefix}_spheres"], G[f"{prefix}_nodes"],
                        G[f"{prefix}_materials"], G[f"{prefix}_textures"], G[f"{prefix}_pixels"],
                        int(G[f"{prefix}_root"]), int(G[f"{prefix}_max_depth"]))


def rel_l2(a, b):
    return float(np.sqrt(((a.astype(np.float64) - b) ** 2).sum() / max(1e-20, (b.astype(np.float64) ** 2).sum())))


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


@pytest.mark.parametrize("prefix,w,h,seed,batches", [("cornell", 32, 20, 1, [2, 1]), ("sphere", 19, 13, 7, [3, 5]),
                                                     ("light0", 19, 13, 11, [16]), ("light1", 19, 13, 11, [16])])
def test_depth50_vs_reference_golden(prefix, w, h, seed, batches):
    """Against the reference's CPU renderer (golden sums), depth 50 as the reference hard-codes."""
    s = golden_scene(prefix)
    r = pt.CudaRenderer(s, G[f"{prefix}_camera"], w, h, seed, max_depth=50)
    for b in batches:
        r.add_samples(b)
    key = {"cornell": "cornell_render_mis1", "sphere": "sphere_render"}.get(prefix, prefix)
    want = G[f"{key}_sums"]
    assert rel_l2(r.sums(), want) < REL_L2
    assert r.rays_traced() == int(G[f"{key}_rays"])
    if prefix in ("cornell", "sphere"):
        assert np.array_equal(r.rng_state(), G[f"{key}_rng"])


@pytest.mark.parametrize("mis", [True, False])
@pytest.mark.parametrize("depth", [8, 50])
def test_cornell_vs_oracle(oracle, mis, depth):
    s, cam = pt.cornell_box(80, 50)
    r = pt.CudaRenderer(s, cam, 80, 50, 1, direct_light=mis, max_depth=depth)
    r.add_samples(3)
    r.add_samples(1)
    sums, rng, rays = oracle.render(s, cam, 80, 50, 1, [3, 1], max_depth=depth, mis=mis)
    assert rel_l2(r.sums(), sums) < REL_L2
    assert r.rays_traced() == rays
    assert np.array_equal(r.rng_state(), rng)


@pytest.mark.parametrize("debug", range(1, 6))
def test_debug_views_vs_golden(debug):
    s = golden_scene("cornell")
    r = pt.CudaRenderer(s, G["cornell_camera"], 32, 20, 1, debug=debug)
    r.add_samples(2)
    assert rel_l2(r.sums(), G[f"cornell_debug{debug}_sums"]) < REL_L2
    assert r.rays_traced() == int(G[f"cornell_debug{debug}_rays"])


def test_progressive_batching_is_byte_stable():
    s, cam = pt.cornell_box(40, 25)
    a = pt.CudaRenderer(s, cam, 40, 25, 7, max_depth=8)
    b = pt.CudaRenderer(s, cam, 40, 25, 7, max_depth=8)
    a.add_samples(7)
    b.add_samples(2)
    b.add_samples(1)
    b.add_samples(4)
    assert a.sums().tobytes() == b.sums().tobytes()
    assert a.rays_traced() == b.rays_traced()
    b.reset(cam)
    assert b.sample_count() == 0 and not b.sums().any() and b.rays_traced() == 0
    b.add_samples(7)
    assert a.sums().tobytes() == b.sums().tobytes()


def test_brute_matches_bvh():
    s, cam = pt.cornell_box(40, 25)
    a = pt.CudaRenderer(s, cam, 40, 25, 3, max_depth=8)
    b = pt.CudaRenderer(s, cam, 40, 25, 3, brute=True, max_depth=8)
    a.add_samples(4)
    b.add_samples(4)
    assert rel_l2(b.sums(), a.sums()) < REL_L2


def test_block_shapes_and_argument_errors():
    s, cam = pt.cornell_box(24, 16)
    r = pt.CudaRenderer(s, cam, 24, 16, 3, max_depth=8)
    base = pt.CudaRenderer(s, cam, 24, 16, 3, max_depth=8)
    base.add_samples(2)
    for shape in [(8, 8), (16, 8), (16, 16), (32, 8)]:
        r.set_block_shape(*shape)
    r.add_samples(2)
    assert r.sums().tobytes() == base.sums().tobytes()
    with pytest.raises(ValueError):
        r.set_block_shape(3, 3)
    with pytest.raises(ValueError):
        r.add_samples(0)
    with pytest.raises(ValueError):
        pt.CudaRenderer(s, cam, 0, 16, 3)
    with pytest.raises(ValueError):
        pt.CudaRenderer(s, cam, 24, 16, 3, debug=9)
    bad = cam.copy()
    bad["lens_radius"] = -1
    with pytest.raises(ValueError):
        r.reset(bad)


def test_rgba_packing(oracle):
    s, cam = pt.cornell_box(24, 16)
    r = pt.CudaRenderer(s, cam, 24, 16, 3, max_depth=8)
    r.add_samples(4)
    got = r.rgba_image()
    assert np.array_equal(got, oracle.pack_rgba(r.sums(), 4, host_image=False))
    host = oracle.pack_rgba(r.sums(), 4, host_image=True)
    assert np.abs(got.astype(int) - host.astype(int)).max() <= 1   # tests/lighting_tests.cpp:93-94


@pytest.mark.skipif(not REF_GPU_SO.exists(), reason="reference CUDA build absent")
@pytest.mark.parametrize("debug", [0, 1, 2, 3, 4, 5])
def test_bit_identical_to_reference_gpu_renderer(debug):
    """The reference's own cuda_renderer, built for sm_100a, on the same B200."""
    s = golden_scene("sphere")
    cam = G["sphere_camera"]
    ref = RefGpu().renderer(s, cam, 19, 13, 7, debug=debug)
    ref.add_samples(3)
    ref.add_samples(5)
    ours = pt.CudaRenderer(s, cam, 19, 13, 7, debug=debug, max_depth=50)
    ours.add_samples(3)
    ours.add_samples(5)
    assert ours.image().tobytes() == ref.image().tobytes()
    assert ours.rays_traced() == ref.stats()[2]
    assert ours.rgba_image().tobytes() == ref.rgba().tobytes()
    ref.close()


@pytest.mark.skipif(not REF_GPU_SO.exists(), reason="reference CUDA build absent")
def test_bit_identical_to_reference_gpu_cornell():
    s, cam = pt.cornell_box(64, 40)
    ref = RefGpu().renderer(s, cam, 64, 40, 1)
    ref.add_samples(4)
    ours = pt.CudaRenderer(s, cam, 64, 40, 1, max_depth=50)
    ours.add_samples(4)
    assert ours.image().tobytes() == ref.image().tobytes()
    assert ours.rays_traced() == ref.stats()[2]
    ref.close()
