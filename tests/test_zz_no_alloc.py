"""The query entry point that allocates nothing (pt_query_rays_static).

Callers that cannot let a library allocate device memory — applications that hand all device
memory to their own pool allocator, latency-critical loops where cudaFree's device-wide
synchronization would stall other streams, processes under a device-memory cap — use this form
instead of pt_query_rays.  It stages through one static device array, so it takes at most
PT_STATIC_QUERY_MAX_RAYS rays per call.  Its answers must equal pt_query_rays's, bit for bit,
call after call (the array keeps the previous call's contents, so a call that forgot to clear
its counter would show up on the second call), and the device's free memory must not change
across calls.  Per-ray counters are compared under the single-loop walk, where a lane's counts
depend only on its own ray (the phased walk lets a lane walk on while its warp searches, so its
counts depend on which rays share the warp).  This file is collected last so that a run that
stops at the first failure has already run every other test; it also passes on its own.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import ptb200 as pt

pytestmark = pytest.mark.gpu
MAX_RAYS = 65536   # PT_STATIC_QUERY_MAX_RAYS in include/pt.h


def static_query(scene: pt.Scene, rays, mode, tmin, tmax, stats: bool):
    lib = pt.library()
    fn = lib.pt_query_rays_static
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    hits = np.zeros(len(rays), pt.HIT)
    st = np.zeros(len(rays), pt.RAY_STATS) if stats else None
    status = fn(scene.handle, rays.ctypes.data, len(rays), mode, tmin,
                None if tmax is None else tmax.ctypes.data, hits.ctypes.data,
                None if st is None else st.ctypes.data, None)
    return status, hits, st


@pytest.mark.parametrize("speculative", [1, 0])
@pytest.mark.parametrize("mode", [pt.QUERY_CLOSEST, pt.QUERY_ANY])
def test_static_query_matches_allocating_query_twice(mode, speculative):
    import torch
    scene, cam = pt.procedural_scene(96, 60, sphere_count=4, segments=64, rings=33, seed=5)
    dev = pt.Scene(scene)
    batches = [pt.camera_rays(cam, 96, 60, 11 + call, 0, n) for call, n in enumerate((MAX_RAYS, 20000, 777))]
    pt.query_walk(speculative)
    try:
        free = []
        for call, rays in enumerate(batches):
            tmax = None if mode == pt.QUERY_CLOSEST else np.full(len(rays), 12.0, np.float32)
            want, want_stats = dev.query(rays, mode=mode, tmin=0.001, tmax=tmax, stats=True)   # allocates
            torch.cuda.synchronize()
            free.append(torch.cuda.mem_get_info()[0])
            status, hits, stats = static_query(dev, rays, mode, 0.001, tmax, stats=True)
            assert status == 0, pt.library().pt_last_error()
            assert hits.tobytes() == want.tobytes(), f"call {call}"
            if not speculative:
                assert stats.tobytes() == want_stats.tobytes(), f"call {call}"
            assert (hits["primitive_type"] != 0).any()
        # the first call may load the library's device code (and with it the static array); the
        # calls after it allocate nothing
        assert free[1] == free[2], f"free device memory changed across calls: {free}"
    finally:
        pt.query_walk(1)


def test_static_query_rejects_more_than_its_scratch_holds():
    scene, cam = pt.cornell_box(32, 20)
    dev = pt.Scene(scene)
    rays = pt.camera_rays(cam, 32, 20, 1, 0, MAX_RAYS + 1)
    status, _, _ = static_query(dev, rays, pt.QUERY_CLOSEST, 0.001, None, stats=False)
    assert status == 1
    assert "at most 65536 rays" in pt.library().pt_last_error().decode()
