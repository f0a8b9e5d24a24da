"""The radiance-cache renderer: plain mode equals the plain renderer, the cache path is
deterministic and graph-safe, and the trained network beats both the plain path tracer and an
untrained network on the same frame budget.

relMSE = mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2), r = a high-sample plain render.
"""
from __future__ import annotations

import numpy as np
import pytest

import ptb200 as pt

pytestmark = pytest.mark.gpu


def rel_mse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref * ref + 1e-2)))


@pytest.fixture(scope="module")
def cornell():
    flat, camera = pt.cornell_box(96, 64)
    return pt.Scene(flat), camera


@pytest.fixture(scope="module")
def reference(cornell):
    """4096-spp plain render, accumulated in float64 over 16 independent seeds."""
    scene, camera = cornell
    acc = np.zeros((64, 96, 3))
    for k in range(16):
        r = pt.CudaRenderer(scene, camera, 96, 64, seed=1000 + k, max_depth=8)
        r.add_samples(256)
        acc += r.sums().astype(np.float64).reshape(64, 96, 3)
    return acc / 4096


def test_plain_mode_equals_plain_renderer(cornell):
    """use_cache=0: the same MIS estimator, consuming every pixel's PCG stream in the same
    order, so the sums equal the plain renderer's up to float rounding of the products."""
    scene, camera = cornell
    plain = pt.CudaRenderer(scene, camera, 96, 64, seed=3, max_depth=8)
    plain.add_samples(16)
    cached = pt.CachedRenderer(scene, camera, 96, 64, seed=3, max_depth=8, use_cache=0, samples_per_frame=4)
    cached.frames(4)
    a, b = cached.sums().astype(np.float64).reshape(-1), plain.sums().astype(np.float64).reshape(-1)
    np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-4)
    st = cached.stats()
    assert st["frames"] == 16 and st["queries"] == 0 and st["samples"] == 0
    assert abs(st["rays"] - plain.rays_traced()) <= 0.001 * plain.rays_traced()


def test_samples_per_frame_are_frames_in_one_launch(cornell):
    """A pixel's samples run one after the other inside a frame, consuming its PCG stream and
    adding to its sum in the order separate frames would."""
    scene, camera = cornell
    one = pt.CachedRenderer(scene, camera, 96, 64, seed=9, max_depth=8, use_cache=0, samples_per_frame=1)
    one.frames(8)
    eight = pt.CachedRenderer(scene, camera, 96, 64, seed=9, max_depth=8, use_cache=0, samples_per_frame=8)
    eight.frames(1)
    assert one.sums().tobytes() == eight.sums().tobytes()
    assert one.stats()["frames"] == eight.stats()["frames"] == 8


def test_graph_and_launches_agree_with_frozen_network(cornell):
    """train=0: no training, so the frame is deterministic; the captured graph and the
    one-by-one launches give the same bits."""
    scene, camera = cornell
    out = []
    for graph in (1, 0):
        r = pt.CachedRenderer(scene, camera, 96, 64, seed=5, max_depth=8, train=0, use_graph=graph)
        r.frames(4)
        out.append(r.sums())
        st = r.stats()
        assert st["queries"] > 0 and st["samples"] == 0
    assert out[0].tobytes() == out[1].tobytes()


def test_training_lowers_loss(cornell):
    """The median of the last-step losses over 15 frames falls with training (single steps are
    noisy: a batch can hold a path that found the light through a mirror)."""
    scene, camera = cornell
    r = pt.CachedRenderer(scene, camera, 96, 64, seed=7, max_depth=8, training_paths=2048)

    def median_loss():
        out = []
        for _ in range(15):
            r.train(1)
            out.append(r.stats()["loss"])
        return float(np.median(out))

    early = median_loss()
    r.train(300)
    late = median_loss()
    assert r.stats()["samples"] > 0 and np.isfinite(late)
    assert late < 0.5 * early, (early, late)


def test_trained_cache_gains_over_plain_and_untrained(cornell, reference):
    """Same frame count: the trained cache has lower relMSE than the plain path tracer and
    than the same renderer with its network left untrained."""
    scene, camera = cornell
    frames = 16                                     # x 4 samples per frame
    plain = pt.CachedRenderer(scene, camera, 96, 64, seed=11, max_depth=8, use_cache=0)
    plain.frames(frames)
    untrained = pt.CachedRenderer(scene, camera, 96, 64, seed=11, max_depth=8, train=0)
    untrained.frames(frames)
    trained = pt.CachedRenderer(scene, camera, 96, 64, seed=11, max_depth=8, training_paths=1024)
    trained.train(400)
    trained.frames(frames)
    e_plain, e_untrained, e_trained = (rel_mse(r.image(), reference) for r in (plain, untrained, trained))
    print(f"relMSE at {4 * frames} samples: plain {e_plain:.3e}, untrained cache {e_untrained:.3e}, trained cache {e_trained:.3e}")
    assert e_trained < e_plain
    assert e_trained < 0.5 * e_untrained


def test_rejects_bad_settings(cornell):
    scene, camera = cornell
    for bad in (dict(train_steps=0), dict(train_steps=9), dict(suffix_bounces=0), dict(suffix_bounces=9),
                dict(training_paths=-1), dict(learning_rate=0.0), dict(spread_threshold=-1.0),
                dict(tail_paths=-1), dict(samples_per_frame=0), dict(samples_per_frame=65),
                dict(weight_average=1.0)):
        with pytest.raises(ValueError):
            pt.CachedRenderer(scene, camera, 8, 8, **bad)
    with pytest.raises(ValueError):
        pt.CachedRenderer(scene, camera, 8, 8, train=0).train(1)   # training-only frames need training
    with pytest.raises(TypeError):
        pt.CachedRenderer(scene, camera, 8, 8, no_such_setting=1)
