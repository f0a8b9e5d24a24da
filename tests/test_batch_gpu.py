"""Batched rendering: many jobs in one graph launch give each job the bits of a lone renderer."""
from __future__ import annotations

import numpy as np
import pytest

import ptb200 as pt

pytestmark = pytest.mark.gpu


def make_jobs():
    cornell, ccam = pt.cornell_box(48, 30)
    proc, pcam = pt.procedural_scene(40, 25, sphere_count=3, segments=48, rings=25, seed=4)
    proc2, pcam2 = pt.procedural_scene(64, 36, sphere_count=2, segments=32, rings=17, seed=9, floor=0)
    scenes = [cornell, proc, proc2]
    jobs = [dict(scene=0, camera=ccam, width=48, height=30, samples=5, max_depth=8, seed=1),
            dict(scene=1, camera=pcam, width=40, height=25, samples=3, max_depth=12, seed=2),
            dict(scene=2, camera=pcam2, width=64, height=36, samples=4, max_depth=4, seed=3),
            dict(scene=0, camera=ccam, width=48, height=30, samples=2, max_depth=50, seed=4)]
    return scenes, jobs


def alone(scenes, job, mis=True):
    r = pt.CudaRenderer(scenes[job["scene"]], job["camera"], job["width"], job["height"], job["seed"],
                        direct_light=mis, max_depth=job["max_depth"])
    r.add_samples(job["samples"])
    return r.sums(), r.rays_traced()


@pytest.mark.parametrize("wide", [1, 0], ids=["four-wide", "two-wide"])
@pytest.mark.parametrize("graph", [1, 0], ids=["graph", "host-loop"])
@pytest.mark.parametrize("capacity", [0, 700], ids=["all-slots", "small-pool"])
def test_batch_matches_lone_renderers(graph, capacity, wide):
    scenes, jobs = make_jobs()
    b = pt.Batch(scenes, jobs)
    b.tuning(path_capacity=capacity, use_graph=graph)
    b.node_width(wide)
    b.run()
    ms, rays, done = b.stats()
    total = 0
    for k, j in enumerate(jobs):
        want, r = alone(scenes, j)
        total += r
        assert b.sums(k).tobytes() == want.tobytes(), f"job {k}"
    assert rays == total
    assert (done > 0).all() and (done <= ms * 1.05 + 0.5).all()
    b.run()   # a second run starts from a fresh state
    for k, j in enumerate(jobs):
        assert b.sums(k).tobytes() == alone(scenes, j)[0].tobytes()


def test_batch_classic_lighting_and_tail_modes():
    scenes, jobs = make_jobs()
    b = pt.Batch(scenes, jobs, direct_light=False)
    for tail in (0, 1 << 30):
        b.tuning(tail_paths=tail)
        b.run()
        for k, j in enumerate(jobs):
            assert b.sums(k).tobytes() == alone(scenes, j, mis=False)[0].tobytes()


def test_batch_autotune_caches(tmp_path):
    scenes, jobs = make_jobs()
    b = pt.Batch(scenes, jobs)
    cache = tmp_path / "batch_tuning.txt"
    best = b.autotune(probe_samples=1, cache_path=str(cache))
    assert cache.exists() and len(cache.read_text().splitlines()) == 1
    assert best[1] in (128, 256) and best[3] in (0, 1)
    again = b.autotune(probe_samples=1, cache_path=str(cache))   # served from the cache
    assert again == best and len(cache.read_text().splitlines()) == 1
    b.run()
    for k, j in enumerate(jobs):
        assert b.sums(k).tobytes() == alone(scenes, j)[0].tobytes()


def test_batch_rejects_bad_jobs():
    scenes, jobs = make_jobs()
    bad = dict(jobs[0], scene=7)
    with pytest.raises(ValueError):
        pt.Batch(scenes, [bad])
    with pytest.raises(ValueError):
        pt.Batch(scenes, [dict(jobs[0], samples=0)])


@pytest.mark.parametrize("fail_at", [1, 5])
def test_autotune_skips_a_failed_probe_and_keeps_sample_counts(fail_at):
    """A probe run that fails (injected on the host as a timed-out run) skips its setting; the
    sweep goes on, and afterwards every job renders its full sample count."""
    scenes, jobs = make_jobs()
    b = pt.Batch(scenes, jobs)
    pt.check(pt.library().pt_batch_fail_probe(b._h, fail_at))
    best = b.autotune(probe_samples=1, cache_path=None)
    assert best[1] in (128, 256) and best[4] in (0, 1)
    b.run()
    for k, j in enumerate(jobs):
        assert b.sums(k).tobytes() == alone(scenes, j)[0].tobytes(), f"job {k}"
