"""ctypes bindings of the CPU oracle and of the reference builds — TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs.

* ``Oracle``  — oracle/liboracle.so, the C restatement (oracle/pt_oracle.c).
* ``RefCpu``  — oracle/_ref/libref_cpu.so, the reference's own host code (built from its sources).
* ``RefGpu``  — oracle/_ref/libref_cuda.so, the reference's own CUDA renderer for sm_100a.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "cuda-path-tracer_b200"))
import ptb200 as pt  # noqa: E402
ORACLE_SO = ROOT / "oracle" / "liboracle.so"
REF_CPU_SO = ROOT / "oracle" / "_ref" / "libref_cpu.so"
REF_GPU_SO = ROOT / "oracle" / "_ref" / "libref_cuda.so"
P, S, I, U64, F = C.c_void_p, C.c_size_t, C.c_int, C.c_uint64, C.c_float


class View(C.Structure):
    """or_view (oracle/pt_oracle.h) — scene_view of the reference."""
    _fields_ = [("triangles", P), ("spheres", P), ("nodes", P), ("materials", P), ("textures", P), ("pixels", P),
                ("root", C.c_int32), ("node_count", C.c_int32), ("lights", P), ("light_count", C.c_int32),
                ("light_area", C.c_float)]


def threads() -> int:
    return max(1, os.cpu_count() or 1)


class Oracle:
    def __init__(self):
        if not ORACLE_SO.exists():
            raise RuntimeError("oracle/liboracle.so is not built (make -C oracle oracle)")
        lib = C.CDLL(str(ORACLE_SO))
        sig = {
            "or_validate": (I, [P]),
            "or_scene_lights": (S, [P, P, S, P, P]),
            "or_rng_seed": (None, [P, U64, U64]),
            "or_rng_next": (C.c_uint32, [P]),
            "or_rng_uniform": (F, [P]),
            "or_trace_box": (I, [P, P, F, F]),
            "or_triangle_hit": (I, [P, P, F, F, P]),
            "or_sphere_hit": (I, [P, P, F, F, P]),
            "or_trace_world": (I, [P, P, F, F, P, I, I, P, P, P]),
            "or_query": (None, [P, P, S, I, F, P, I, I, P, P, I]),
            "or_query_ties": (None, [P, P, S, I, F, P, I, I, P, P, P, I]),
            "or_query_compat": (None, [P, P, S, I, P, I]),
            "or_add_samples": (I, [P, P, I, I, I, I, I, I, I, P, P, P, I]),
            "or_reset": (None, [I, I, U64, P, P]),
            "or_pack_rgba": (None, [P, S, I, I, P]),
            "or_image": (None, [P, S, I, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        self.lib = lib

    # -- scene view (keeps references alive on the object)
    def view(self, scene: pt.FlatScene, with_lights: bool = True):
        lights, area = self.lights(scene) if with_lights else (np.zeros(0, pt.LIGHT), 0.0)
        v = View()
        v.triangles, v.spheres, v.nodes = _p(scene.triangles), _p(scene.spheres), _p(scene.nodes)
        v.materials, v.textures, v.pixels = _p(scene.materials), _p(scene.textures), _p(scene.pixels)
        v.root, v.node_count = scene.root, len(scene.nodes)
        v.lights, v.light_count, v.light_area = _p(lights), len(lights), area
        v._keep = (scene, lights)
        return v

    def validate(self, scene: pt.FlatScene) -> bool:
        d = scene.desc()
        return self.lib.or_validate(C.byref(d)) == 0

    def lights(self, scene: pt.FlatScene):
        d = scene.desc()
        area, status = C.c_float(), C.c_int()
        n = self.lib.or_scene_lights(C.byref(d), None, 0, C.byref(area), C.byref(status))
        out = np.zeros(n, pt.LIGHT)
        self.lib.or_scene_lights(C.byref(d), _p(out), n, C.byref(area), C.byref(status))
        if status.value:
            raise ValueError("light area exceeds range")
        return out, area.value

    def query(self, scene, rays, mode=pt.QUERY_CLOSEST, tmin=0.001, tmax=None, brute=False, tie_lowest=True,
              stats=False, nthreads=None):
        v = self.view(scene, with_lights=False)
        rays = np.ascontiguousarray(rays, pt.RAY)
        hits = np.zeros(len(rays), pt.HIT)
        st = np.zeros(len(rays), pt.RAY_STATS) if stats else None
        tm = None if tmax is None else np.ascontiguousarray(tmax, np.float32)
        self.lib.or_query(C.byref(v), _p(rays), len(rays), mode, tmin, _p(tm), int(brute), int(tie_lowest), _p(hits),
                          _p(st), nthreads or threads())
        return (hits, st) if stats else hits

    def query_ties(self, scene, rays, mode=pt.QUERY_CLOSEST, tmin=0.001, tmax=None, nthreads=None):
        """Closest (lowest-id ties) or any hit, plus per ray how many other primitives were hit
        at exactly the closest distance: (hits, ties)."""
        v = self.view(scene, with_lights=False)
        rays = np.ascontiguousarray(rays, pt.RAY)
        hits = np.zeros(len(rays), pt.HIT)
        ties = np.zeros(len(rays), np.int32)
        tm = None if tmax is None else np.ascontiguousarray(tmax, np.float32)
        self.lib.or_query_ties(C.byref(v), _p(rays), len(rays), mode, tmin, _p(tm), 0, 1, _p(hits), None, _p(ties),
                               nthreads or threads())
        return hits, ties

    def query_compat(self, scene, rays, brute=False):
        v = self.view(scene, with_lights=False)
        rays = np.ascontiguousarray(rays, pt.RAY)
        out = np.zeros(len(rays), pt.TRACE_RESULT)
        self.lib.or_query_compat(C.byref(v), _p(rays), len(rays), int(brute), _p(out), threads())
        return out

    def render(self, scene, camera, width, height, seed, batches, max_depth=50, debug=0, mis=True, brute=False,
               nthreads=None):
        """Progressive render: reset, then add_samples(b) for b in batches.  Returns (sums, rng, rays)."""
        v = self.view(scene)
        sums = np.zeros(width * height * 3, np.float32)
        rng = np.zeros(width * height * 2, np.uint64)
        self.lib.or_reset(width, height, seed, _p(sums), _p(rng))
        rays = C.c_uint64(0)
        cam = np.ascontiguousarray(camera, pt.CAMERA)
        for b in batches:
            err = self.lib.or_add_samples(C.byref(v), _p(cam), width, height, b, int(brute), debug, int(mis), max_depth,
                                          _p(sums), _p(rng), C.byref(rays), nthreads or threads())
            if err:
                raise RuntimeError("portable traversal stack overflow")
        return sums, rng, rays.value

    def image(self, sums, samples):
        out = np.zeros_like(sums)
        self.lib.or_image(_p(sums), len(sums) // 3, samples, _p(out))
        return out

    def pack_rgba(self, sums, samples, host_image=False):
        out = np.zeros(len(sums) // 3 * 4, np.uint8)
        self.lib.or_pack_rgba(_p(sums), len(sums) // 3, samples, int(host_image), _p(out))
        return out

    def rng_draws(self, seed, pixel, count):
        st = (C.c_uint64 * 2)()
        self.lib.or_rng_seed(st, seed, pixel)
        return np.array([self.lib.or_rng_uniform(st) for _ in range(count)], np.float32)


class RefCpu:
    """The reference's own host code, compiled from its sources into oracle/_ref/."""

    def __init__(self):
        if not REF_CPU_SO.exists():
            raise RuntimeError("oracle/_ref/libref_cpu.so is not built (make -C oracle ref)")
        lib = C.CDLL(str(REF_CPU_SO))
        sig = {
            "ref_validate": (I, [P]),
            "ref_scene_lights": (I, [P, P, S, P, P]),
            "ref_trace_world_batch": (I, [P, P, S, F, P, I, P, P, I]),
            "ref_render": (I, [P, P, I, I, I, I, I, I, P, P, P, I]),
            "ref_reset_pixels": (None, [I, I, U64, P, P]),
            "ref_portable_image": (I, [P, P, I, I, U64, I, I, I, P, I, P, P]),
            "ref_display_pixels": (None, [P, S, P]),
            "ref_rng_draws": (None, [U64, U64, I, P, P]),
            "ref_triangle_hit": (I, [P, P, F, F, P]),
            "ref_sphere_hit": (I, [P, P, F, F, P]),
            "ref_trace_box": (I, [P, P, F, F]),
            "ref_flat_mesh": (P, [P, P, P, I, C.c_long]),
            "ref_flat_obj": (P, [C.c_char_p, I, I, P, P, P, C.c_long, C.c_char_p, S]),
            "ref_camera": (None, [P, P, P, F, F, F, F, F, F, P]),
            "ref_flat_counts": (None, [P, P, P, P]),
            "ref_flat_copy": (None, [P, P, P, P, P, P, P, P]),
            "ref_flat_free": (None, [P]),
            "ref_mesh_create": (P, [P, S, C.c_long]),
            "ref_mesh_hit": (None, [P, P, S, F, P, I]),
            "ref_mesh_free": (None, [P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        self.lib = lib

    def validate(self, scene) -> bool:
        d = scene.desc()
        return self.lib.ref_validate(C.byref(d)) == 0

    def lights(self, scene):
        d = scene.desc()
        n, area = C.c_size_t(), C.c_float()
        if self.lib.ref_scene_lights(C.byref(d), None, 0, C.byref(n), C.byref(area)):
            raise ValueError("light area exceeds range")
        out = np.zeros(n.value, pt.LIGHT)
        self.lib.ref_scene_lights(C.byref(d), _p(out), n.value, C.byref(n), C.byref(area))
        return out, area.value

    def trace_world(self, scene, rays, tmin=0.001, tmax=None, brute=False, nthreads=None):
        d = scene.desc()
        rays = np.ascontiguousarray(rays, pt.RAY)
        out = np.zeros(len(rays), pt.TRACE_RESULT)
        st = np.zeros(len(rays), pt.RAY_STATS)
        tm = None if tmax is None else np.ascontiguousarray(tmax, np.float32)
        self.lib.ref_trace_world_batch(C.byref(d), _p(rays), len(rays), tmin, _p(tm), int(brute), _p(out), _p(st),
                                       nthreads or threads())
        return out, st

    def render(self, scene, camera, width, height, seed, batches, debug=0, mis=True, brute=False, nthreads=None):
        """trace_pixel_sample per pixel at the reference's depth 50.  Returns (sums, rng, rays)."""
        d = scene.desc()
        sums = np.zeros(width * height * 3, np.float32)
        rng = np.zeros(width * height * 2, np.uint64)
        self.lib.ref_reset_pixels(width, height, seed, _p(sums), _p(rng))
        rays = C.c_uint64(0)
        cam = np.ascontiguousarray(camera, pt.CAMERA)
        for b in batches:
            err = self.lib.ref_render(C.byref(d), _p(cam), width, height, b, int(brute), debug, int(mis), _p(sums),
                                      _p(rng), C.byref(rays), nthreads or threads())
            if err:
                raise RuntimeError(f"reference render failed ({err})")
        return sums, rng, rays.value

    def portable_image(self, scene, camera, width, height, seed, batches, debug=0, mis=True, brute=False):
        d = scene.desc()
        b = np.asarray(batches, np.int32)
        img = np.zeros(width * height * 3, np.float32)
        rays = C.c_uint64(0)
        cam = np.ascontiguousarray(camera, pt.CAMERA)
        if self.lib.ref_portable_image(C.byref(d), _p(cam), width, height, seed, int(brute), debug, int(mis), _p(b),
                                       len(b), _p(img), C.byref(rays)):
            raise RuntimeError("reference portable renderer failed")
        return img, rays.value

    def display_pixels(self, rgb):
        out = np.zeros(len(rgb) // 3 * 4, np.uint8)
        self.lib.ref_display_pixels(_p(np.ascontiguousarray(rgb, np.float32)), len(rgb) // 3, _p(out))
        return out

    def rng_draws(self, seed, pixel, count):
        u = np.zeros(count, np.float32)
        raw = np.zeros(count, np.uint32)
        self.lib.ref_rng_draws(seed, pixel, count, _p(u), _p(raw))
        return u, raw

    def _take(self, h) -> pt.FlatScene:
        counts = (C.c_size_t * 6)()
        root, depth = C.c_int32(), C.c_int32()
        self.lib.ref_flat_counts(h, counts, C.byref(root), C.byref(depth))
        s = pt.FlatScene(np.zeros(counts[0], pt.TRIANGLE), np.zeros(counts[1], pt.SPHERE), np.zeros(counts[2], pt.NODE),
                         np.zeros(counts[3], pt.MATERIAL), np.zeros(counts[4], pt.TEXTURE),
                         np.zeros(counts[5], np.uint8), root.value, depth.value)
        cam = np.zeros(1, pt.CAMERA)
        self.lib.ref_flat_copy(h, _p(s.triangles), _p(s.spheres), _p(s.nodes), _p(s.materials), _p(s.textures),
                               _p(s.pixels), _p(cam))
        self.lib.ref_flat_free(h)
        return s, cam

    def flat_mesh(self, vertices, colors, kinds, seed=7) -> pt.FlatScene:
        """triangle_mesh(faces) flattened by the reference (random-axis bvh_node after srand48(seed))."""
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3, 3)
        c = np.ascontiguousarray(colors, np.float32).reshape(-1, 3)
        k = np.ascontiguousarray(kinds, np.int32)
        h = self.lib.ref_flat_mesh(_p(v), _p(c), _p(k), len(v), seed)
        if not h:
            raise RuntimeError("reference flatten failed")
        return self._take(h)[0]

    def flat_obj(self, path, width, height, scale=(1, 1, 1), rotate=(0, 0, 0), translate=(0, 0, 0), seed=7):
        """The CLI's scene pipeline (src/app/main.cpp:27-32): (flat scene, camera)."""
        f = lambda v: (C.c_float * 3)(*v)
        err = C.create_string_buffer(512)
        h = self.lib.ref_flat_obj(str(path).encode(), width, height, f(scale), f(rotate), f(translate), seed, err, 512)
        if not h:
            raise RuntimeError(err.value.decode())
        return self._take(h)

    def camera(self, lookfrom, lookat, vup, vfov, aspect, aperture, focus, t0, t1):
        f = lambda v: (C.c_float * 3)(*v)
        out = np.zeros(1, pt.CAMERA)
        self.lib.ref_camera(f(lookfrom), f(lookat), f(vup), vfov, aspect, aperture, focus, t0, t1, _p(out))
        return out

    def mesh_hit(self, vertices, rays, seed=7, tmin=0.001, nthreads=None):
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3, 3)
        h = self.lib.ref_mesh_create(_p(v), len(v), seed)
        try:
            rays = np.ascontiguousarray(rays, pt.RAY)
            t = np.zeros(len(rays), np.float32)
            self.lib.ref_mesh_hit(h, _p(rays), len(rays), tmin, _p(t), nthreads or threads())
            return t
        finally:
            self.lib.ref_mesh_free(h)


class RefMesh:
    """The reference's pre-CUDA host path: its triangle objects under its own bvh_node (random-axis
    median split, drand48 seeded), hit through the virtual hittable::hit, as
    tests/mesh_validation.cpp:76-81 does.  Built once; hits() timed separately."""

    def __init__(self, ref: RefCpu, vertices, seed: int = 7):
        self.ref = ref
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3, 3)
        self.h = ref.lib.ref_mesh_create(_p(v), len(v), seed)
        if not self.h:
            raise RuntimeError("ref_mesh_create failed")

    def hits(self, rays, tmin=0.001, nthreads=None):
        """t of the closest hit per ray (-1 on a miss)."""
        rays = np.ascontiguousarray(rays, pt.RAY)
        t = np.zeros(len(rays), np.float32)
        self.ref.lib.ref_mesh_hit(self.h, _p(rays), len(rays), tmin, _p(t), nthreads or threads())
        return t

    def close(self):
        if self.h:
            self.ref.lib.ref_mesh_free(self.h)
            self.h = None


REF_TIMING_SO = REF_GPU_SO.with_name("libref_cuda_timing.so")


class RefGpuTiming:
    """Device time of the reference's own query_rays kernel (oracle/ref_cuda_timing.cu): the scene
    uploaded by its device_scene, rays already on the device, CUDA events around the launches."""

    def __init__(self):
        if not REF_TIMING_SO.exists():
            raise RuntimeError(f"{REF_TIMING_SO} is not built (make -C oracle ref)")
        lib = C.CDLL(str(REF_TIMING_SO))
        lib.reftime_last_error.restype, lib.reftime_last_error.argtypes = C.c_char_p, []
        lib.reftime_query.restype = I
        lib.reftime_query.argtypes = [P, P, S, I, I, P, P, S]
        self.lib = lib

    def query(self, scene, device_rays: int, count: int, warmup: int = 1, reps: int = 3, sample: int = 0):
        """(mean kernel ms, the first `sample` trace_result records of the last launch)."""
        d = scene.desc()
        ms = C.c_float()
        out = np.zeros(sample, pt.TRACE_RESULT)
        if self.lib.reftime_query(C.byref(d), device_rays, count, warmup, reps, C.byref(ms), _p(out), sample):
            raise RuntimeError(self.lib.reftime_last_error().decode())
        return ms.value, out


def ref_gpu_so(depth=None) -> Path:
    """oracle/_ref/libref_cuda.so, or the patched build whose bounce limit is `depth` (8 or 12)."""
    return REF_GPU_SO if depth is None else REF_GPU_SO.with_name(f"libref_cuda_d{depth}.so")


class RefGpu:
    """The reference's own CUDA renderer and cuda_query_rays (sm_100a build).  depth=8 or 12
    loads the "patched reference": the same sources with trace_color's bounce limit of 50
    (src/renderer/transport.h:174,193) set to that depth (oracle/Makefile)."""

    def __init__(self, depth=None):
        so = ref_gpu_so(depth)
        if not so.exists():
            raise RuntimeError(f"{so} is not built (make -C oracle ref)")
        lib = C.CDLL(str(so))
        sig = {
            "refgpu_last_error": (C.c_char_p, []),
            "refgpu_available": (I, [C.c_char_p, S]),
            "refgpu_query": (I, [P, P, S, I, P]),
            "refgpu_renderer_create": (P, [P, P, I, I, U64, I, I, I]),
            "refgpu_add_samples": (I, [P, I]),
            "refgpu_set_block_shape": (I, [P, I, I]),
            "refgpu_reset": (I, [P, P]),
            "refgpu_image": (I, [P, P]),
            "refgpu_rgba": (I, [P, P]),
            "refgpu_stats": (None, [P, P, P, P]),
            "refgpu_destroy": (None, [P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        self.lib = lib

    def _check(self, rc):
        if rc:
            raise RuntimeError(self.lib.refgpu_last_error().decode())

    def query(self, scene, rays, brute=False):
        d = scene.desc()
        rays = np.ascontiguousarray(rays, pt.RAY)
        out = np.zeros(len(rays), pt.TRACE_RESULT)
        self._check(self.lib.refgpu_query(C.byref(d), _p(rays), len(rays), int(brute), _p(out)))
        return out

    def renderer(self, scene, camera, width, height, seed, brute=False, debug=0, mis=True):
        d = scene.desc()
        cam = np.ascontiguousarray(camera, pt.CAMERA)
        h = self.lib.refgpu_renderer_create(C.byref(d), _p(cam), width, height, seed, int(brute), debug, int(mis))
        if not h:
            raise RuntimeError(self.lib.refgpu_last_error().decode())
        return RefGpuRenderer(self, h, width * height)


class RefGpuRenderer:
    def __init__(self, owner, h, pixels):
        self.o, self.h, self.pixels = owner, h, pixels

    def add_samples(self, n):
        self.o._check(self.o.lib.refgpu_add_samples(self.h, n))

    def set_block_shape(self, w, h):
        self.o._check(self.o.lib.refgpu_set_block_shape(self.h, w, h))

    def image(self):
        out = np.zeros(self.pixels * 3, np.float32)
        self.o._check(self.o.lib.refgpu_image(self.h, _p(out)))
        return out

    def rgba(self):
        out = np.zeros(self.pixels * 4, np.uint8)
        self.o._check(self.o.lib.refgpu_rgba(self.h, _p(out)))
        return out

    def stats(self):
        s, ms, r = C.c_int(), C.c_float(), C.c_uint64()
        self.o.lib.refgpu_stats(self.h, C.byref(s), C.byref(ms), C.byref(r))
        return s.value, ms.value, r.value

    def close(self):
        if self.h:
            self.o.lib.refgpu_destroy(self.h)
            self.h = None


def _p(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data if a.size else None
    return a
