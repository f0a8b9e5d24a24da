"""GPU parity of the wavefront renderer against the oracle and the reference's own renderer.

Bars:
* against the reference's CUDA renderer on the same B200 (same arithmetic, same CUDA math
  functions): linear sums, RGBA bytes and ray counts are bit-identical;
* against the CPU oracle / the reference's CPU renderer: CUDA's cosf/sinf/powf/atan2f differ from
  glibc's by a few ULP, so a small fraction of paths take a different turn (the reference's own
  GPU build shows the same against its CPU build, see test_reference_gpu_vs_cpu_is_statistical).
  Once a path diverges, that pixel's PCG stream is shifted for all of its later samples, so on
  long closed-box paths (depth 50) a sizeable fraction of pixels differ.  The bar is
  statistical: the mean per-pixel difference is within 4 standard errors of zero (a z-test on
  the per-pixel differences), fewer than half the pixels differ, and ray counts agree to 1 %.  On scenes without that sensitivity
  the reference's own bar (relative L2 < 1e-4 with equal ray counts, tests/lighting_tests.cpp:86-92)
  holds and is asserted.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import ptb200 as pt
from oracle_bind import Oracle, RefGpu, REF_GPU_SO, ref_gpu_so

pytestmark = pytest.mark.gpu
G = np.load(Path(__file__).parent / "golden" / "reference_golden.npz")
REL_L2 = 1e-4


def golden_scene(prefix):
    return pt.FlatScene(G[f"{prefix}_triangles"], G[f"{prefix}_spheres"], G[f"{prefix}_nodes"],
                        G[f"{prefix}_materials"], G[f"{prefix}_textures"], G[f"{prefix}_pixels"],
                        int(G[f"{prefix}_root"]), int(G[f"{prefix}_max_depth"]))


def assert_statistically_equal(gpu_sums, cpu_sums, spp, gpu_rays, cpu_rays):
    a = gpu_sums.reshape(-1, 3).astype(np.float64) / spp
    b = cpu_sums.reshape(-1, 3).astype(np.float64) / spp
    differs = (np.abs(a - b) > 1e-5 * np.maximum(1, np.abs(b))).any(axis=1)
    assert differs.mean() < 0.5, differs.mean()
    d = (a - b).mean(axis=1)
    se = d.std() / np.sqrt(len(d))
    assert abs(d.mean()) <= 4 * se + 1e-7, (d.mean(), se)
    assert abs(int(gpu_rays) - int(cpu_rays)) <= 0.01 * cpu_rays, (gpu_rays, cpu_rays)


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
    if prefix == "cornell":      # closed box at depth 50: long paths, some diverge (see module doc)
        assert_statistically_equal(r.sums(), want, sum(batches), r.rays_traced(), int(G[f"{key}_rays"]))
        return
    assert rel_l2(r.sums(), want) < REL_L2
    assert r.rays_traced() == int(G[f"{key}_rays"])
    if prefix == "sphere":
        assert np.array_equal(r.rng_state(), G[f"{key}_rng"])


@pytest.mark.parametrize("mis", [True, False])
@pytest.mark.parametrize("depth", [8, 50])
def test_cornell_vs_oracle(oracle, mis, depth):
    s, cam = pt.cornell_box(80, 50)
    r = pt.CudaRenderer(s, cam, 80, 50, 1, direct_light=mis, max_depth=depth)
    r.add_samples(3)
    r.add_samples(1)
    sums, rng, rays = oracle.render(s, cam, 80, 50, 1, [3, 1], max_depth=depth, mis=mis)
    assert_statistically_equal(r.sums(), sums, 4, r.rays_traced(), rays)
    same = (r.rng_state().reshape(-1, 2) == rng.reshape(-1, 2)).all(axis=1)
    assert same.mean() >= (0.98 if depth == 8 else 0.5)   # a diverged path shifts its pixel's stream


@pytest.mark.parametrize("debug", range(1, 6))
def test_debug_views_vs_golden(debug):
    s = golden_scene("cornell")
    r = pt.CudaRenderer(s, G["cornell_camera"], 32, 20, 1, debug=debug)
    r.add_samples(2)
    assert rel_l2(r.sums(), G[f"cornell_debug{debug}_sums"]) < REL_L2   # debug views stop at the first hit
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
@pytest.mark.parametrize("tail", [0, None, 2**31 - 1], ids=["wavefront", "hybrid", "fused"])
@pytest.mark.parametrize("wide", [1, 0], ids=["wide", "binary"])
def test_bit_identical_to_reference_gpu_cornell(tail, wide):
    """Pure wavefront, the default hybrid and the fused finish kernel, on either node layout, all
    give the reference's bits."""
    pt.query_layout(wide)
    s, cam = pt.cornell_box(64, 40)
    ref = RefGpu().renderer(s, cam, 64, 40, 1)
    ref.add_samples(4)
    ours = pt.CudaRenderer(s, cam, 64, 40, 1, max_depth=50)
    if tail is not None:
        ours.set_tail_paths(tail)
    ours.add_samples(4)
    pt.query_layout(1)
    assert ours.image().tobytes() == ref.image().tobytes()
    assert ours.rays_traced() == ref.stats()[2]
    ref.close()


@pytest.mark.parametrize("depth", [8, 12])
def test_bit_identical_to_patched_reference_at_depth(depth):
    """The configs quoted at bounce limits 8 and 12 against the "patched reference" (the same
    renderer sources with the literal 50 set to that depth): the same bits, on the Cornell box and
    a small procedural scene, MIS and classic lighting."""
    if not ref_gpu_so(depth).exists():
        pytest.skip("patched reference build absent")
    scenes = [pt.cornell_box(64, 40), pt.procedural_scene(48, 30, sphere_count=3, segments=48, rings=25, seed=4)]
    for (s, cam), mis in zip(scenes, (True, False)):
        w, h = (64, 40) if len(s.spheres) else (48, 30)
        ref = RefGpu(depth).renderer(s, cam, w, h, 3, mis=mis)
        ref.add_samples(5)
        ours = pt.CudaRenderer(s, cam, w, h, 3, direct_light=mis, max_depth=depth)
        ours.add_samples(5)
        assert ours.image().tobytes() == ref.image().tobytes()
        assert ours.rays_traced() == ref.stats()[2]
        ref.close()


@pytest.mark.parametrize("tail", [0, 2**31 - 1], ids=["wavefront", "fused"])
@pytest.mark.parametrize("debug", [0, 4, 5])
def test_tail_modes_agree(tail, debug):
    s, cam = pt.cornell_box(48, 30)
    a = pt.CudaRenderer(s, cam, 48, 30, 5, max_depth=8, debug=debug)
    a.add_samples(3)
    b = pt.CudaRenderer(s, cam, 48, 30, 5, max_depth=8, debug=debug)
    b.set_tail_paths(tail)
    b.add_samples(3)
    assert a.sums().tobytes() == b.sums().tobytes() and a.rays_traced() == b.rays_traced()
    assert a.rng_state().tobytes() == b.rng_state().tobytes()


@pytest.mark.skipif(not REF_GPU_SO.exists(), reason="reference CUDA build absent")
def test_reference_gpu_vs_cpu_is_statistical():
    """The reference's own GPU renderer against its own CPU path on the golden Cornell render:
    the same few-ULP transcendental differences make a few paths diverge, so the statistical bar
    above is the reference's own GPU-vs-CPU behaviour, not a weakening for the new kernels."""
    s = golden_scene("cornell")
    ref = RefGpu().renderer(s, G["cornell_camera"], 32, 20, 1)
    ref.add_samples(2)
    ref.add_samples(1)
    spp, _, rays = ref.stats()
    img = ref.image()
    ref.close()
    cpu = G["cornell_render_mis1_sums"] * np.float32(1.0 / 3)
    assert_statistically_equal(img, cpu, 1, rays, int(G["cornell_render_mis1_rays"]))
