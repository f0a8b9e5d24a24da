"""ptb200 — Python binding of the B200 path-tracing core (libptb200.so, C ABI in include/pt.h).

Mirrors the reference renderer surface of AdmiralHeathCL/cuda-path-tracer:

* ``cuda_device_available()``            — src/cuda/cuda_renderer.h:8
* ``CudaRenderer``                        — class cuda_renderer, src/cuda/cuda_renderer.h:10-29
* ``obj_scene``                           — load_obj + obj_scene, src/scene/obj_loader.h, obj_scene.h
* ``cuda_query_rays(scene, rays, brute)`` — src/cuda/cuda_renderer.h:32
* numpy record dtypes with the byte layout of the flat transfer records (src/flat/flat_data.h).

Errors raise the exception types the reference throws: ``ValueError`` for its
``std::invalid_argument`` and ``RuntimeError`` for its ``std::runtime_error``.  There is no
CPU fallback: without the compiled library or a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIBRARY_PATH = _HERE.parent / "libptb200.so"

# ---------------------------------------------------------------- record dtypes (pt.h)
VEC3 = ("<f4", (3,))
TRIANGLE = np.dtype([("v0", *VEC3), ("v1", *VEC3), ("v2", *VEC3), ("n0", *VEC3), ("n1", *VEC3), ("n2", *VEC3),
                     ("uv0", *VEC3), ("uv1", *VEC3), ("uv2", *VEC3), ("material_id", "<i4"), ("smooth", "<i4")])
SPHERE = np.dtype([("center", *VEC3), ("radius", "<f4"), ("material_id", "<i4")])
NODE = np.dtype([("minimum", *VEC3), ("maximum", *VEC3), ("type", "<i4"), ("left", "<i4"), ("right", "<i4"),
                 ("primitive", "<i4")])
MATERIAL = np.dtype([("albedo", *VEC3), ("fuzz", "<f4"), ("ref_idx", "<f4"), ("type", "<i4"), ("texture_id", "<i4")])
TEXTURE = np.dtype([("color", *VEC3), ("scale", *VEC3), ("offset", *VEC3), ("type", "<i4"), ("image_id", "<i4"),
                    ("width", "<i4"), ("height", "<i4"), ("byte_offset", "<i4"), ("clamp", "<i4")])
CAMERA = np.dtype([("origin", *VEC3), ("lower_left_corner", *VEC3), ("horizontal", *VEC3), ("vertical", *VEC3),
                   ("u", *VEC3), ("v", *VEC3), ("lens_radius", "<f4"), ("time0", "<f4"), ("time1", "<f4")])
RAY = np.dtype([("origin", *VEC3), ("direction", *VEC3), ("time", "<f4")])
FLAT_HIT = np.dtype([("t", "<f4"), ("u", "<f4"), ("v", "<f4"), ("p", *VEC3), ("normal", *VEC3),
                     ("material_id", "<i4"), ("primitive_type", "<i4"), ("primitive_id", "<i4")])
TRACE_RESULT = np.dtype([("rec", FLAT_HIT), ("hit", "<i4"), ("error", "<i4")])
LIGHT = np.dtype([("type", "<i4"), ("primitive", "<i4"), ("cumulative_area", "<f4")])
HIT = np.dtype([("t", "<f4"), ("primitive_id", "<i4"), ("primitive_type", "<i4"), ("error", "<i4")])
RAY_STATS = np.dtype([("boxes", "<u4"), ("primitives", "<u4")])
for _name, _dt, _size in [("triangle", TRIANGLE, 116), ("sphere", SPHERE, 20), ("node", NODE, 40),
                          ("material", MATERIAL, 28), ("texture", TEXTURE, 60), ("camera", CAMERA, 84),
                          ("ray", RAY, 28), ("flat_hit", FLAT_HIT, 48), ("trace_result", TRACE_RESULT, 56),
                          ("light", LIGHT, 12), ("hit", HIT, 16)]:
    assert _dt.itemsize == _size, (_name, _dt.itemsize)

BRANCH, TRIANGLE_TYPE, SPHERE_TYPE = 0, 1, 2
DIFFUSE, METAL, GLASS, LIGHT_MAT = 0, 1, 2, 3
TEX_CONSTANT, TEX_IMAGE, TEX_MAP = 0, 1, 2
DEBUG_SHADED, DEBUG_NORMALS, DEBUG_TRIANGLE, DEBUG_MATERIAL, DEBUG_BVH, DEBUG_INTERSECTIONS = range(6)
QUERY_CLOSEST, QUERY_ANY = 0, 1
RENDER_MIS, RENDER_BRUTE = 1, 2

STATUS = {0: "PT_OK", 1: "PT_INVALID_ARGUMENT", 2: "PT_INVALID_SCENE", 3: "PT_CUDA_ERROR",
          4: "PT_STACK_OVERFLOW", 5: "PT_QUEUE_OVERFLOW", 6: "PT_TIMEOUT", 7: "PT_NO_DEVICE"}


class PtError(RuntimeError):
    """A failing pt_* call; ``status`` is the pt_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class PtInvalidArgument(PtError, ValueError):
    """PT_INVALID_ARGUMENT — the reference's std::invalid_argument."""


class _SceneDesc(C.Structure):
    _fields_ = [("triangles", C.c_void_p), ("triangle_count", C.c_size_t),
                ("spheres", C.c_void_p), ("sphere_count", C.c_size_t),
                ("nodes", C.c_void_p), ("node_count", C.c_size_t),
                ("materials", C.c_void_p), ("material_count", C.c_size_t),
                ("textures", C.c_void_p), ("texture_count", C.c_size_t),
                ("pixels", C.c_void_p), ("pixel_bytes", C.c_size_t),
                ("root", C.c_int32), ("max_depth", C.c_int32)]


class ProceduralParams(C.Structure):
    """pt_procedural_params (include/pt_workloads.h)."""
    _fields_ = [("sphere_count", C.c_int), ("segments", C.c_int), ("rings", C.c_int), ("box_size", C.c_float),
                ("displacement", C.c_float), ("radius_min", C.c_float), ("radius_max", C.c_float),
                ("floor", C.c_int), ("light_fraction", C.c_float), ("light_radiance", C.c_float),
                ("metal_fraction", C.c_float), ("glass_fraction", C.c_float), ("seed", C.c_uint64),
                ("random_triangles", C.c_int), ("soup_edge_min", C.c_float), ("soup_edge_max", C.c_float),
                ("gpu_bvh", C.c_int)]


_lib = None


def library() -> C.CDLL:
    """Loads libptb200.so (built by __graft_entry__.build() / make -C cuda-path-tracer_b200)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY_PATH.exists():
        raise RuntimeError(f"libptb200.so is not built ({LIBRARY_PATH}); run make -C cuda-path-tracer_b200")
    lib = C.CDLL(str(LIBRARY_PATH))
    P, S, I, U64, F = C.c_void_p, C.c_size_t, C.c_int, C.c_uint64, C.c_float
    sig = {
        "pt_device_available": (I, [C.c_char_p, S]),
        "pt_last_error": (C.c_char_p, []),
        "pt_abi_version": (I, []),
        "pt_scene_create": (I, [P, P]),
        "pt_scene_destroy": (I, [P]),
        "pt_scene_lights": (I, [P, P, S, P, P]),
        "pt_scene_device_bytes": (I, [P, P]),
        "pt_query_ordered": (I, [P, S, P]),
        "pt_layout_check": (I, [P, P, P]),
        "pt_query_rays_device": (I, [P, P, S, I, F, P, P, P, P]),
        "pt_query_rays_brute_device": (I, [P, P, S, I, F, P, P, P, P]),
        "pt_query_rays": (I, [P, P, S, I, F, P, P, P]),
        "pt_query_rays_compat": (I, [P, P, S, I, P]),
        "pt_query_tuning": (I, [I, I, I]),
        "pt_query_layout": (I, [I]),
        "pt_query_walk": (I, [I]),
        "pt_query_order": (I, [I]),
        "pt_query_profile": (I, [P, I]),
        "pt_query_profile_read": (I, [P, P, S, P]),
        "pt_probe_read_bandwidth": (I, [S, I, P]),
        "pt_rays_camera_device": (I, [P, I, I, U64, U64, S, P, P]),
        "pt_rays_bounce_device": (I, [P, P, P, S, U64, U64, P, P]),
        "pt_rays_surface_device": (I, [P, U64, U64, S, P, P, P]),
        "pt_rays_camera_at": (I, [P, I, I, U64, P, S, P]),
        "pt_rays_bounce_at": (I, [P, P, P, S, U64, P, P, I]),
        "pt_flat_from_desc": (I, [P, P]),
        "pt_flat_build_bvh": (I, [P, I]),
        "pt_flat_desc": (I, [P, P]),
        "pt_flat_destroy": (I, [P]),
        "pt_make_camera": (I, [P, P, P, F, F, F, F, F, F, P]),
        "pt_workload_cornell": (I, [I, I, P, P]),
        "pt_procedural_defaults": (None, [P]),
        "pt_workload_procedural": (I, [P, I, I, P, P]),
        "pt_workload_obj": (I, [C.c_char_p, I, I, P, P, P, P, P, P, S]),
        "pt_flat_build_bvh_gpu": (I, [P]),
        "pt_rays_camera": (I, [P, I, I, U64, U64, S, P]),
        "pt_rays_surface": (I, [P, U64, U64, S, P, P, I]),
        "pt_rays_bounce": (I, [P, P, P, S, U64, U64, P, I]),
        "pt_renderer_create": (I, [P, P, I, I, U64, C.c_uint32, I, I, P]),
        "pt_renderer_destroy": (I, [P]),
        "pt_reset": (I, [P, P]),
        "pt_add_samples": (I, [P, I]),
        "pt_set_block_shape": (I, [P, I, I]),
        "pt_get_sums": (I, [P, P, S]),
        "pt_get_image": (I, [P, P, S]),
        "pt_get_rng": (I, [P, P, S]),
        "pt_write_rgba": (I, [P, P, S]),
        "pt_rgba_image": (I, [P, P, S]),
        "pt_stats": (I, [P, P, P, P]),
        "pt_renderer_tuning": (I, [P, C.c_int32]),
        "pt_batch_create": (I, [P, C.c_int32, P, C.c_int32, C.c_uint32, P]),
        "pt_batch_destroy": (I, [P]),
        "pt_batch_run": (I, [P]),
        "pt_batch_get_sums": (I, [P, C.c_int32, P, S]),
        "pt_batch_stats": (I, [P, P, P, P, S]),
        "pt_batch_tuning": (I, [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
        "pt_batch_autotune": (I, [P, C.c_int32, C.c_char_p, P]),
        "pt_batch_fail_probe": (I, [P, C.c_int32]),
        "pt_batch_node_width": (I, [P, C.c_int32]),
        "pt_cache_create": (I, [P, P, U64, P]),
        "pt_cache_destroy": (I, [P]),
        "pt_cache_query_device": (I, [P, P, S, P, P]),
        "pt_cache_train_device": (I, [P, P, P, S, P, P]),
        "pt_cache_gradients": (I, [P, P, P, S, P, P]),
        "pt_cache_weights": (I, [P, P, P, S]),
        "pt_cache_hyper": (I, [P, F, F, F, F]),
        "pt_cache_average": (I, [P, F]),
        "pt_cache_sync": (I, [P, P]),
        "pt_cache_wait_limit": (I, [P, C.c_longlong]),
        "pt_cached_defaults": (I, [P]),
        "pt_cached_create": (I, [P, P, C.c_int, C.c_int, U64, C.c_int, P, P]),
        "pt_cached_destroy": (I, [P]),
        "pt_cached_frames": (I, [P, C.c_int, C.c_int]),
        "pt_cached_clear": (I, [P]),
        "pt_cached_training": (I, [P, C.c_int]),
        "pt_cached_get_sums": (I, [P, P, S]),
        "pt_cached_stats": (I, [P, P, P, P, P, P, P]),
        "pt_cached_cache": (I, [P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != 0:
        msg = library().pt_last_error().decode(errors="replace")
        if status == 1:
            raise PtInvalidArgument(status, msg)
        raise PtError(status, msg)


def _ptr(a) -> int | None:
    """Address of a numpy array, a torch tensor, an int address or None."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"], "arrays must be contiguous"
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(f"cannot take the address of {type(a)!r}")


def cuda_device_available() -> tuple[bool, str]:
    """cuda_device_available(description) (src/cuda/cuda_renderer.cu:128-140)."""
    buf = C.create_string_buffer(256)
    ok = library().pt_device_available(buf, 256)
    return bool(ok), buf.value.decode(errors="replace")


# ---------------------------------------------------------------- host flat scenes
class FlatScene:
    """Host flat scene (the reference's ``flat_scene``): numpy arrays of the transfer records."""

    def __init__(self, triangles=None, spheres=None, nodes=None, materials=None, textures=None, pixels=None,
                 root=-1, max_depth=0):
        self.triangles = np.ascontiguousarray(triangles if triangles is not None else np.zeros(0, TRIANGLE), TRIANGLE)
        self.spheres = np.ascontiguousarray(spheres if spheres is not None else np.zeros(0, SPHERE), SPHERE)
        self.nodes = np.ascontiguousarray(nodes if nodes is not None else np.zeros(0, NODE), NODE)
        self.materials = np.ascontiguousarray(materials if materials is not None else np.zeros(0, MATERIAL), MATERIAL)
        self.textures = np.ascontiguousarray(textures if textures is not None else np.zeros(0, TEXTURE), TEXTURE)
        self.pixels = np.ascontiguousarray(pixels if pixels is not None else np.zeros(0, np.uint8), np.uint8)
        self.root = int(root)
        self.max_depth = int(max_depth)

    def desc(self) -> _SceneDesc:
        d = _SceneDesc()
        for name in ("triangles", "spheres", "nodes", "materials", "textures", "pixels"):
            arr = getattr(self, name)
            setattr(d, name, arr.ctypes.data if arr.size else None)
        d.triangle_count, d.sphere_count, d.node_count = len(self.triangles), len(self.spheres), len(self.nodes)
        d.material_count, d.texture_count, d.pixel_bytes = len(self.materials), len(self.textures), len(self.pixels)
        d.root, d.max_depth = self.root, self.max_depth
        return d

    def copy(self) -> "FlatScene":
        return FlatScene(self.triangles.copy(), self.spheres.copy(), self.nodes.copy(), self.materials.copy(),
                         self.textures.copy(), self.pixels.copy(), self.root, self.max_depth)

    def build_bvh(self, threads: int = 0, gpu: bool = False) -> "FlatScene":
        """Replaces the nodes with the library's binned-SAH tree (pt_flat_build_bvh), or with
        the linear BVH built on the GPU (gpu=True, pt_flat_build_bvh_gpu)."""
        lib = library()
        h = C.c_void_p()
        d = self.desc()
        check(lib.pt_flat_from_desc(C.byref(d), C.byref(h)))
        try:
            check(lib.pt_flat_build_bvh_gpu(h) if gpu else lib.pt_flat_build_bvh(h, threads))
            return _flat_from_handle(h)
        finally:
            lib.pt_flat_destroy(h)

    def save(self, path) -> None:
        np.savez_compressed(path, triangles=self.triangles, spheres=self.spheres, nodes=self.nodes,
                            materials=self.materials, textures=self.textures, pixels=self.pixels,
                            root=self.root, max_depth=self.max_depth)

    @staticmethod
    def load(path) -> "FlatScene":
        z = np.load(path)
        return FlatScene(z["triangles"], z["spheres"], z["nodes"], z["materials"], z["textures"], z["pixels"],
                         int(z["root"]), int(z["max_depth"]))


def _flat_from_handle(h) -> FlatScene:
    d = _SceneDesc()
    check(library().pt_flat_desc(h, C.byref(d)))

    def grab(ptr, count, dtype):
        out = np.zeros(count, dtype)
        if count:
            C.memmove(out.ctypes.data, ptr, count * dtype.itemsize)
        return out
    return FlatScene(grab(d.triangles, d.triangle_count, TRIANGLE), grab(d.spheres, d.sphere_count, SPHERE),
                     grab(d.nodes, d.node_count, NODE), grab(d.materials, d.material_count, MATERIAL),
                     grab(d.textures, d.texture_count, TEXTURE), grab(d.pixels, d.pixel_bytes, np.dtype(np.uint8)),
                     d.root, d.max_depth)


def make_camera(lookfrom, lookat, vup=(0, 1, 0), vfov=40.0, aspect=1.0, aperture=0.0, focus_dist=1.0,
                time0=0.0, time1=1.0) -> np.ndarray:
    """The reference camera (src/core/camera.h:16-43), flattened."""
    out = np.zeros(1, CAMERA)
    f = lambda v: (C.c_float * 3)(*v)
    check(library().pt_make_camera(f(lookfrom), f(lookat), f(vup), vfov, aspect, aperture, focus_dist, time0, time1,
                                   out.ctypes.data))
    return out


def cornell_box(width: int = 320, height: int = 200) -> tuple[FlatScene, np.ndarray]:
    """The 20-triangle Cornell-style box with three spheres (pt_workload_cornell)."""
    lib = library()
    h = C.c_void_p()
    cam = np.zeros(1, CAMERA)
    check(lib.pt_workload_cornell(width, height, C.byref(h), cam.ctypes.data))
    try:
        return _flat_from_handle(h), cam
    finally:
        lib.pt_flat_destroy(h)


def procedural_params(**overrides) -> ProceduralParams:
    p = ProceduralParams()
    library().pt_procedural_defaults(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def layout_check(flat: "FlatScene") -> tuple[int, int]:
    """(four-wide nodes, violations) of the tree pt_scene_create would build (pt_layout_check; host only)."""
    d = flat.desc()
    nodes, bad = C.c_size_t(), C.c_size_t()
    check(library().pt_layout_check(C.byref(d), C.byref(nodes), C.byref(bad)))
    return nodes.value, bad.value


def procedural_scene(width: int = 960, height: int = 600, **overrides) -> tuple[FlatScene, np.ndarray]:
    """Displaced-sphere scene (pt_workload_procedural); defaults = the 1M-triangle scene."""
    lib = library()
    p = procedural_params(**overrides)
    h = C.c_void_p()
    cam = np.zeros(1, CAMERA)
    check(lib.pt_workload_procedural(C.byref(p), width, height, C.byref(h), cam.ctypes.data))
    try:
        return _flat_from_handle(h), cam
    finally:
        lib.pt_flat_destroy(h)


def obj_scene(path, width: int, height: int, scale=(1, 1, 1), rotate=(0, 0, 0), translate=(0, 0, 0)):
    """OBJ/MTL import and the reference's preview stage (pt_workload_obj): (FlatScene, camera,
    warnings) for a width x height render, as `ray_tracer --obj path` sets it up."""
    lib = library()
    h = C.c_void_p()
    cam = np.zeros(1, CAMERA)
    f = lambda v: (C.c_float * 3)(*[float(x) for x in v])
    warn = C.create_string_buffer(4096)
    check(lib.pt_workload_obj(str(path).encode(), width, height, f(scale), f(rotate), f(translate), C.byref(h),
                              cam.ctypes.data, warn, 4096))
    try:
        return _flat_from_handle(h), cam, warn.value.decode()
    finally:
        lib.pt_flat_destroy(h)


def camera_rays(camera: np.ndarray, width: int, height: int, seed: int, first: int, count: int) -> np.ndarray:
    out = np.zeros(count, RAY)
    check(library().pt_rays_camera(camera.ctypes.data, width, height, seed, first, count, out.ctypes.data))
    return out


def camera_rays_at(camera: np.ndarray, width: int, height: int, seed: int, index) -> np.ndarray:
    """The camera rays of camera_rays with the given ray indices (pt_rays_camera_at)."""
    index = np.ascontiguousarray(index, np.uint64)
    out = np.zeros(len(index), RAY)
    check(library().pt_rays_camera_at(camera.ctypes.data, width, height, seed, _ptr(index), len(index), _ptr(out)))
    return out


def surface_rays(scene: FlatScene, seed: int, first: int, count: int, shadow: bool = False, threads: int = 0):
    lib = library()
    h = C.c_void_p()
    d = scene.desc()
    check(lib.pt_flat_from_desc(C.byref(d), C.byref(h)))
    try:
        rays = np.zeros(count, RAY)
        tmax = np.zeros(count, np.float32) if shadow else None
        check(lib.pt_rays_surface(h, seed, first, count, rays.ctypes.data, _ptr(tmax), threads))
        return (rays, tmax) if shadow else rays
    finally:
        lib.pt_flat_destroy(h)


def bounce_rays(scene: FlatScene, primary: np.ndarray, hits: np.ndarray, seed: int, first: int,
                threads: int = 0) -> np.ndarray:
    """Host bounce rays (pt_rays_bounce), bit-identical to Scene.bounce_rays_device."""
    lib = library()
    h = C.c_void_p()
    d = scene.desc()
    check(lib.pt_flat_from_desc(C.byref(d), C.byref(h)))
    try:
        primary = np.ascontiguousarray(primary, RAY)
        hits = np.ascontiguousarray(hits, HIT)
        out = np.zeros(len(primary), RAY)
        check(lib.pt_rays_bounce(h, _ptr(primary), _ptr(hits), len(primary), seed, first, _ptr(out), threads))
        return out
    finally:
        lib.pt_flat_destroy(h)


def bounce_rays_at(scene: FlatScene, primary: np.ndarray, hits: np.ndarray, seed: int, streams,
                   threads: int = 0) -> np.ndarray:
    """bounce_rays with an explicit PCG stream index per ray (pt_rays_bounce_at)."""
    lib = library()
    h = C.c_void_p()
    d = scene.desc()
    check(lib.pt_flat_from_desc(C.byref(d), C.byref(h)))
    try:
        primary = np.ascontiguousarray(primary, RAY)
        hits = np.ascontiguousarray(hits, HIT)
        streams = np.ascontiguousarray(streams, np.uint64)
        out = np.zeros(len(primary), RAY)
        check(lib.pt_rays_bounce_at(h, _ptr(primary), _ptr(hits), len(primary), seed, _ptr(streams), _ptr(out), threads))
        return out
    finally:
        lib.pt_flat_destroy(h)


# ---------------------------------------------------------------- device scene + queries
class Scene:
    """Device-resident scene (pt_scene_create): validated, re-laid out and uploaded."""

    def __init__(self, flat: FlatScene):
        self.flat = flat
        self._h = C.c_void_p()
        d = flat.desc()
        check(library().pt_scene_create(C.byref(d), C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            library().pt_scene_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def lights(self):
        n = C.c_size_t()
        area = C.c_float()
        check(library().pt_scene_lights(self._h, None, 0, C.byref(n), C.byref(area)))
        out = np.zeros(n.value, LIGHT)
        check(library().pt_scene_lights(self._h, _ptr(out), n.value, C.byref(n), C.byref(area)))
        return out, area.value

    def device_bytes(self) -> int:
        n = C.c_size_t()
        check(library().pt_scene_device_bytes(self._h, C.byref(n)))
        return n.value

    def query_ordered(self, count: int) -> bool:
        """Whether a query of `count` rays is walked in key order under the current settings (pt_query_ordered)."""
        o = C.c_int()
        check(library().pt_query_ordered(self._h, int(count), C.byref(o)))
        return bool(o.value)

    def query(self, rays: np.ndarray, mode: int = QUERY_CLOSEST, tmin: float = 0.001, tmax=None, stats=False):
        """Host-buffer query (pt_query_rays): returns HIT records (and RAY_STATS)."""
        rays = np.ascontiguousarray(rays, RAY)
        hits = np.zeros(len(rays), HIT)
        st = np.zeros(len(rays), RAY_STATS) if stats else None
        tm = None if tmax is None else np.ascontiguousarray(tmax, np.float32)
        check(library().pt_query_rays(self._h, _ptr(rays), len(rays), mode, tmin, _ptr(tm), _ptr(hits), _ptr(st)))
        return (hits, st) if stats else hits

    def query_device(self, rays, count: int, hits, mode: int = QUERY_CLOSEST, tmin: float = 0.001, tmax=None,
                     stats=None, stream=0, brute=False):
        """Device-buffer query (pt_query_rays_device); arguments are device addresses or tensors."""
        fn = library().pt_query_rays_brute_device if brute else library().pt_query_rays_device
        check(fn(self._h, _ptr(rays), count, mode, tmin, _ptr(tmax), _ptr(hits), _ptr(stats), stream))

    def query_compat(self, rays: np.ndarray, brute: bool = False) -> np.ndarray:
        rays = np.ascontiguousarray(rays, RAY)
        out = np.zeros(len(rays), TRACE_RESULT)
        check(library().pt_query_rays_compat(self._h, _ptr(rays), len(rays), int(brute), _ptr(out)))
        return out

    def profile(self, launches: int) -> None:
        """Records CUDA events around the next walk-kernel launches (a ring of `launches`; 0 stops)."""
        check(library().pt_query_profile(self._h, launches))

    def profile_read(self) -> np.ndarray:
        """Durations (ms) of the walk launches recorded since profile(), oldest first."""
        n = C.c_size_t()
        check(library().pt_query_profile_read(self._h, None, 0, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        check(library().pt_query_profile_read(self._h, _ptr(out), n.value, C.byref(n)))
        return out

    def bounce_rays_device(self, primary, hits, count: int, seed: int, first: int, out, stream=0):
        check(library().pt_rays_bounce_device(self._h, _ptr(primary), _ptr(hits), count, seed, first, _ptr(out), stream))


    def surface_rays_device(self, seed: int, first: int, count: int, out, tmax=None, stream=0):
        """Surface rays (or, with tmax, shadow rays between surface points) on the device."""
        check(library().pt_rays_surface_device(self._h, seed, first, count, _ptr(out), _ptr(tmax), stream))


def camera_rays_device(camera: np.ndarray, width, height, seed, first, count, out, stream=0):
    check(library().pt_rays_camera_device(camera.ctypes.data, width, height, seed, first, count, _ptr(out), stream))


def read_bandwidth(nbytes: int, reps: int = 20) -> float:
    """GB/s of 16-byte loads over a buffer of nbytes (pt_probe_read_bandwidth)."""
    g = C.c_float()
    check(library().pt_probe_read_bandwidth(nbytes, reps, C.byref(g)))
    return g.value


def query_tuning(persistent: int = 1, min_active: int = 24, blocks_per_sm: int = 0) -> None:
    """Sets the ray-query kernel variant and its tunables (pt_query_tuning)."""
    check(library().pt_query_tuning(persistent, min_active, blocks_per_sm))


def query_layout(wide: int = 1) -> None:
    """Four-wide (1) or two-wide (0) node layout for the traversal kernels (pt_query_layout)."""
    check(library().pt_query_layout(int(wide)))


def query_walk(speculative: int = 1) -> None:
    """Four-wide walk form: node/leaf phases (1) or a single loop (0) (pt_query_walk)."""
    check(library().pt_query_walk(int(speculative)))


def query_order(mode: int = 2) -> None:
    """Ray ordering of large batches by (octant, origin Morton code) (pt_query_order): 0 never,
    1 always, 2 when the scene's walked arrays exceed the L2 (default)."""
    check(library().pt_query_order(int(mode)))


def cuda_query_rays(scene: FlatScene, rays: np.ndarray, brute: bool = False) -> np.ndarray:
    """cuda_query_rays(scene, rays, brute) (src/cuda/cuda_renderer.cu:248-260): TRACE_RESULT records."""
    s = Scene(scene)
    try:
        return s.query_compat(rays, brute)
    finally:
        s.close()


# ---------------------------------------------------------------- progressive renderer
class CudaRenderer:
    """class cuda_renderer (src/cuda/cuda_renderer.h:10-29) on the wavefront kernels.

    ``CudaRenderer(scene, camera, width, height, seed, brute=False, debug=DEBUG_SHADED,
    direct_light=True, max_depth=50)``: the reference's constructor arguments plus the bounce
    limit, which the reference hard-codes to 50 (src/renderer/transport.h:174).  ``scene`` is a
    FlatScene (uploaded and owned by the renderer) or a device ``Scene`` (borrowed).
    """

    def __init__(self, scene, camera, width: int, height: int, seed: int, brute: bool = False,
                 debug: int = DEBUG_SHADED, direct_light: bool = True, max_depth: int = 50):
        self._scene = scene if isinstance(scene, Scene) else Scene(scene)
        self.width, self.height = int(width), int(height)
        self._h = C.c_void_p()
        flags = (RENDER_MIS if direct_light else 0) | (RENDER_BRUTE if brute else 0)
        cam = np.ascontiguousarray(camera, CAMERA)
        check(library().pt_renderer_create(self._scene.handle, cam.ctypes.data, self.width, self.height, seed, flags,
                                           debug, max_depth, C.byref(self._h)))

    @property
    def pixels(self) -> int:
        return self.width * self.height

    def close(self):
        if self._h:
            library().pt_renderer_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self, camera) -> None:
        cam = np.ascontiguousarray(camera, CAMERA)
        check(library().pt_reset(self._h, cam.ctypes.data))

    def add_samples(self, count: int) -> None:
        check(library().pt_add_samples(self._h, int(count)))

    def set_block_shape(self, width: int, height: int) -> None:
        check(library().pt_set_block_shape(self._h, width, height))

    def set_tail_paths(self, tail_paths: int) -> None:
        """Live-path count below which the fused finish kernel takes over (pt_renderer_tuning)."""
        check(library().pt_renderer_tuning(self._h, int(tail_paths)))

    def sums(self) -> np.ndarray:
        """Linear FP32 radiance sums, 3 per pixel, not divided by the sample count."""
        out = np.zeros(self.pixels * 3, np.float32)
        check(library().pt_get_sums(self._h, out.ctypes.data, out.size))
        return out

    def image(self) -> np.ndarray:
        out = np.zeros(self.pixels * 3, np.float32)
        check(library().pt_get_image(self._h, out.ctypes.data, out.size))
        return out

    def rng_state(self) -> np.ndarray:
        out = np.zeros(self.pixels * 2, np.uint64)
        check(library().pt_get_rng(self._h, out.ctypes.data, out.size))
        return out

    def rgba_image(self) -> np.ndarray:
        out = np.zeros(self.pixels * 4, np.uint8)
        check(library().pt_rgba_image(self._h, out.ctypes.data, out.size))
        return out

    def write_rgba(self, device_pixels, nbytes: int) -> None:
        check(library().pt_write_rgba(self._h, _ptr(device_pixels), nbytes))

    def _stats(self):
        s, ms, r = C.c_int(), C.c_float(), C.c_uint64()
        check(library().pt_stats(self._h, C.byref(s), C.byref(ms), C.byref(r)))
        return s.value, ms.value, r.value

    def sample_count(self) -> int:
        return self._stats()[0]

    def kernel_milliseconds(self) -> float:
        return self._stats()[1]

    def rays_traced(self) -> int:
        return self._stats()[2]


# ---------------------------------------------------------------- batched rendering
JOB = np.dtype([("scene", "<i4"), ("width", "<i4"), ("height", "<i4"), ("samples", "<i4"), ("max_depth", "<i4"),
                ("pad", "<i4"), ("seed", "<u8"), ("camera", CAMERA), ("tail", "<u4")])
assert JOB.itemsize == 120, JOB.itemsize


class Batch:
    """Many render jobs in one launch (pt_batch_*).  ``jobs`` are dicts with keys scene (index),
    camera, width, height, samples, max_depth, seed."""

    def __init__(self, scenes, jobs, direct_light: bool = True):
        self._scenes = list(scenes)
        descs = (_SceneDesc * len(self._scenes))(*[s.desc() for s in self._scenes])
        arr = np.zeros(len(jobs), JOB)
        for k, j in enumerate(jobs):
            arr[k]["scene"], arr[k]["width"], arr[k]["height"] = j["scene"], j["width"], j["height"]
            arr[k]["samples"], arr[k]["max_depth"], arr[k]["seed"] = j["samples"], j["max_depth"], j["seed"]
            arr[k]["camera"] = np.asarray(j["camera"], CAMERA).reshape(-1)[0]
        self.jobs = arr
        self._h = C.c_void_p()
        check(library().pt_batch_create(descs, len(self._scenes), arr.ctypes.data, len(arr),
                                        RENDER_MIS if direct_light else 0, C.byref(self._h)))

    def close(self):
        if self._h:
            library().pt_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self) -> None:
        check(library().pt_batch_run(self._h))

    def tuning(self, path_capacity=0, block=256, min_active=16, tail_paths=16384, use_graph=1) -> None:
        check(library().pt_batch_tuning(self._h, path_capacity, block, min_active, tail_paths, use_graph))

    def node_width(self, wide: int) -> None:
        """Four-wide nodes (1) or the two-wide layout (0) for the batch's walks (pt_batch_node_width)."""
        check(library().pt_batch_node_width(self._h, int(wide)))

    def autotune(self, probe_samples: int = 1, cache_path: str | None = None):
        """(capacity, block, min_active, use_graph, node_width) of the fastest probe run (pt_batch_autotune)."""
        best = (C.c_int32 * 5)()
        check(library().pt_batch_autotune(self._h, probe_samples, cache_path.encode() if cache_path else None, best))
        return tuple(best)

    def sums(self, job: int) -> np.ndarray:
        j = self.jobs[job]
        out = np.zeros(int(j["width"]) * int(j["height"]) * 3, np.float32)
        check(library().pt_batch_get_sums(self._h, job, out.ctypes.data, out.size))
        return out

    def stats(self):
        ms, rays = C.c_float(), C.c_uint64()
        done = np.zeros(len(self.jobs), np.float64)
        check(library().pt_batch_stats(self._h, C.byref(ms), C.byref(rays), done.ctypes.data, len(done)))
        return ms.value, rays.value, done


# ---------------------------------------------------------------- radiance cache
CACHE_QUERY = np.dtype([("position", *VEC3), ("direction", *VEC3), ("normal", *VEC3), ("albedo", *VEC3),
                        ("roughness", "<f4")])
assert CACHE_QUERY.itemsize == 52
CACHE_WEIGHTS = 20672


class RadianceCache:
    """The tcgen05 radiance-cache MLP (pt_cache_*).  Query/train take device addresses or torch
    tensors (queries: CACHE_QUERY records, targets/outputs: 3 floats per query)."""

    def __init__(self, scene_lo, scene_hi, seed: int = 1):
        self._h = C.c_void_p()
        self._owner = None
        lo = (C.c_float * 3)(*scene_lo)
        hi = (C.c_float * 3)(*scene_hi)
        check(library().pt_cache_create(lo, hi, seed, C.byref(self._h)))

    @classmethod
    def _borrowed(cls, handle, owner):
        """A view of a network another object owns (kept alive through `owner`)."""
        self = cls.__new__(cls)
        self._h = handle
        self._owner = owner
        return self

    def close(self):
        if self._h and self._owner is None:
            library().pt_cache_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def query(self, queries, count: int, out, stream=0) -> None:
        check(library().pt_cache_query_device(self._h, _ptr(queries), count, _ptr(out), stream))

    def train(self, queries, targets, count: int, stream=0, wait: bool = True):
        """One Adam step; returns the batch's mean loss (wait=False: asynchronous, returns None)."""
        loss = C.c_float()
        check(library().pt_cache_train_device(self._h, _ptr(queries), _ptr(targets), count,
                                              C.byref(loss) if wait else None, stream))
        return loss.value if wait else None

    def gradients(self, queries, targets, count: int):
        g = np.zeros(CACHE_WEIGHTS, np.float32)
        loss = C.c_float()
        check(library().pt_cache_gradients(self._h, _ptr(queries), _ptr(targets), count, g.ctypes.data, C.byref(loss)))
        return loss.value, g

    def weights(self) -> np.ndarray:
        w = np.zeros(CACHE_WEIGHTS, np.float32)
        check(library().pt_cache_weights(self._h, w.ctypes.data, None, CACHE_WEIGHTS))
        return w

    def set_weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, np.float32)
        check(library().pt_cache_weights(self._h, None, w.ctypes.data, CACHE_WEIGHTS))

    def hyper(self, lr=1e-2, beta1=0.9, beta2=0.99, eps=1e-8) -> None:
        check(library().pt_cache_hyper(self._h, lr, beta1, beta2, eps))

    def sync(self, stream=0) -> None:
        """Waits for `stream`; raises PtError (status PT_TIMEOUT) if a tensor-core wait ran out."""
        check(library().pt_cache_sync(self._h, stream))

    def wait_limit(self, attempts: int) -> None:
        """try_wait attempts per bounded wait (< 0: the default; 0: every wait runs out at once)."""
        check(library().pt_cache_wait_limit(self._h, attempts))

    def average(self, decay: float) -> None:
        """Queries use a bias-corrected moving average of the weights (decay 0: the weights)."""
        check(library().pt_cache_average(self._h, decay))


class CachedParams(C.Structure):
    """pt_cached_params (include/pt.h)."""
    _fields_ = [("training_paths", C.c_int32), ("train_steps", C.c_int32), ("suffix_bounces", C.c_int32),
                ("use_cache", C.c_int32), ("train", C.c_int32), ("use_graph", C.c_int32),
                ("spread_threshold", C.c_float), ("learning_rate", C.c_float), ("network_seed", C.c_uint64),
                ("tail_paths", C.c_int32), ("query_specular", C.c_int32),
                ("weight_average", C.c_float), ("samples_per_frame", C.c_int32)]


class CachedRenderer:
    """Path tracing with the learned radiance cache (pt_cached_*): frames of one sample per pixel,
    paths ended at the tcgen05 network after their first wide diffuse bounce, the network trained
    online on the renderer's own training paths.  ``use_cache=False`` is the plain path tracer
    through the same kernels.  No counterpart in the reference."""

    def __init__(self, scene, camera: np.ndarray, width: int, height: int, seed: int = 1, max_depth: int = 12, **params):
        self.scene = scene if isinstance(scene, Scene) else Scene(scene)
        self.width, self.height = width, height
        p = CachedParams()
        check(library().pt_cached_defaults(C.byref(p)))
        for k, v in params.items():
            if k not in dict(CachedParams._fields_):
                raise TypeError(f"unknown radiance-cache setting {k!r}")
            setattr(p, k, int(v) if isinstance(v, bool) else v)
        self.params = p
        self._camera = np.ascontiguousarray(camera, CAMERA)
        self._h = C.c_void_p()
        check(library().pt_cached_create(self.scene.handle, self._camera.ctypes.data, width, height, seed, max_depth,
                                         C.byref(p), C.byref(self._h)))

    def close(self):
        if self._h:
            library().pt_cached_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def frames(self, count: int, accumulate: bool = True) -> None:
        check(library().pt_cached_frames(self._h, count, int(accumulate)))

    def train(self, count: int) -> None:
        """Training-only frames: only the training paths are traced; the image is left alone."""
        self.frames(count, accumulate=False)

    def clear(self) -> None:
        check(library().pt_cached_clear(self._h))

    def training(self, on: bool) -> None:
        """Switch online training off (the network is frozen) or back on."""
        check(library().pt_cached_training(self._h, int(on)))

    def sums(self) -> np.ndarray:
        out = np.zeros((self.height, self.width, 3), np.float32)
        check(library().pt_cached_get_sums(self._h, out.ctypes.data, out.size))
        return out

    def image(self) -> np.ndarray:
        """Mean radiance per pixel over the accumulated frames (float64)."""
        n = self.stats()["frames"]
        return self.sums().astype(np.float64) / max(n, 1)

    def stats(self) -> dict:
        frames = C.c_int()
        ms = C.c_float()
        rays, queries, samples = C.c_uint64(), C.c_uint64(), C.c_uint64()
        loss = C.c_float()
        check(library().pt_cached_stats(self._h, C.byref(frames), C.byref(ms), C.byref(rays), C.byref(queries),
                                        C.byref(samples), C.byref(loss)))
        return dict(frames=frames.value, kernel_ms=ms.value, rays=rays.value, queries=queries.value,
                    samples=samples.value, loss=loss.value)

    def cache(self) -> RadianceCache:
        h = C.c_void_p()
        check(library().pt_cached_cache(self._h, C.byref(h)))
        return RadianceCache._borrowed(h, self)
