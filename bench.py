"""Benchmark: closest-hit rays per second on the procedural 1M-triangle scene.

Workload (one "step"): one closest-hit pass over 2^25 rays of the 1,048,580-triangle procedural
scene (16 displaced spheres of 65,536 triangles, a 2-triangle floor, one emissive quad):
2^24 jittered camera rays of a 960x600 image plus 2^24 cosine-sampled bounce rays leaving their
closest hits, with tmin 0.001 and tmax FLT_MAX as cuda_query_rays uses.  Inputs (940 MB of rays)
are larger than L2, so no flush is needed between steps.

The default run (one GPU) prints one JSON line with the headline number and, beside it:
  parity           a seeded random 2^20-ray subset of the timed rays checked against the CPU
                   oracle (lowest-id ties) and the reference's own trace_world (its tie rule)
  reference_gpu    the reference's own query_rays kernel on the same rays and GPU, and a 2^20-ray
                   slice of pt_query_rays_compat compared bytewise with its cuda_query_rays
  cpu_baseline     the reference's trace_world on all host cores (about 10 s of host work);
  cpu_baseline_bvh_node   its pre-CUDA bvh_node::hit path on a random sample
  c3               the traversal microbenchmark (9,437,184 triangles, 2^25 rays) in closest-hit and
                   any-hit modes, with parity on random subsets and the reference's own query kernel
                   on the same rays
  render_c2        the progressive renderer on config 2 against the reference's CUDA renderer
                   (bounce limit 8) on the same GPU, images compared bitwise
  render_c2_depth50   the same at the reference's own bounce limit 50, against its unpatched build
  render_c1        the Cornell box (config 1) against the reference's CUDA renderer
  cache_c5         the radiance-cache renderer against plain path tracing at 1920x1080: time to
                   the plain method's 1024-spp relMSE and to relMSE <= 1e-3, wall and device time

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--quick]
  python bench.py --workload batch48|cache|mlp|render|c3     one sub-workload as its own line
  python bench.py --workload render --render-scene cornell    the config-1 render alone

--impl reference times the reference's own CPU traversal (trace_world on host_view, built from
its sources into oracle/_ref/) on all host threads over a seeded random sample of the same rays.
Under torchrun every rank traces its own replica of the workload (weak scaling, no collective
on the data path); rank 0 prints one JSON line; the sub-records run only at N=1.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "cuda-path-tracer_b200"))
import ptb200 as pt  # noqa: E402

METRIC = "Grays/s closest-hit"
UNIT = "Grays/s"
WIDTH, HEIGHT = 960, 600
LOG2_RAYS = 25
WORKLOAD = "procedural-1M-triangles closest-hit, 2^24 camera + 2^24 bounce rays"
# CUB's stable radix sort of 30-bit keys: 4 onesweep passes + a histogram + an exclusive sum
SORT_LAUNCHES = 6


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--log2-rays", type=int, default=LOG2_RAYS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--quick", action="store_true", help="headline only: no parity, baselines or sub-records")
    ap.add_argument("--no-c3", action="store_true")
    ap.add_argument("--no-render", action="store_true")
    ap.add_argument("--no-cache", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--parity-rays", type=int, default=1 << 20)
    ap.add_argument("--c3-log2-rays", type=int, default=25)
    ap.add_argument("--dump-rays", default=None,
                    help="directory: write the 2^24 camera and 2^24 bounce rays as raw 28-byte records (the reference's ray layout)")
    ap.add_argument("--workload", choices=["query", "batch48", "cache", "mlp", "render", "c3"], default="query",
                    help="query: the closest-hit benchmark with its sub-records (default); batch48: 48 render jobs in "
                         "one launch; cache: radiance-cache renderer vs plain at 1920x1080; render: config-2 renderer "
                         "vs the reference's; c3: the 9.4M-triangle traversal microbenchmark")
    ap.add_argument("--jobs", type=int, default=48)
    ap.add_argument("--render-scene", choices=["procedural", "cornell"], default="procedural",
                    help="render workload: config 2 (procedural 1M triangles, 960x600, 64 spp) or config 1 (Cornell "
                         "box, 320x200, 16 spp), bounce limit 8")
    ap.add_argument("--ref-spp", type=int, default=65536,
                    help="cache workload: samples of the FP64 reference image (0: time cached frames only)")
    ap.add_argument("--max-spp", type=int, default=4096, help="cache workload: sample budget of each curve")
    ap.add_argument("--bvh", choices=["sah", "lbvh"], default="sah",
                    help="query and batch48 workloads: the host binned-SAH tree (default) or the linear BVH built on the GPU")
    ap.add_argument("--no-graph", action="store_true",
                    help="cache frames: launch the kernels one by one instead of one graph per frame (for profilers)")
    return ap.parse_args(argv)


def measured_peaks():
    """(HBM GB/s, dense BF16 TFLOP/s burst, "measured" | "fallback")."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d.get("bf16_tflops", 1590.0)), "measured"
    return 6650.0, 1590.0, "fallback"


def profile_summary(name: str = "query_walk_ncu.json"):
    """Figures of a committed ncu summary of the walk kernel (profiles/query_walk_ncu.json for
    config 2, profiles/query_microbenchmark_ncu.json for config 3)."""
    p = ROOT / "profiles" / name
    return json.loads(p.read_text()) if p.exists() else {}


def build_scene():
    t = time.perf_counter()
    scene, cam = pt.procedural_scene(WIDTH, HEIGHT)
    return scene, cam, time.perf_counter() - t


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None
        self.dev = device_index
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(device_index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------------ samples
def random_indices(total: int, count: int, seed: int) -> np.ndarray:
    """`count` distinct indices of [0, total), seeded, ascending."""
    g = np.random.default_rng(seed)
    return np.sort(g.choice(total, size=min(count, total), replace=False)).astype(np.uint64)


def reference_sample(scene, cam, per_half: int, ref, seed: int, n_each: int = 1 << (LOG2_RAYS - 1)):
    """A seeded random sample of the benchmark's rays built on the host: `per_half` camera rays at
    random indices of the 2^24 camera rays, and the bounce rays of `per_half` other random camera
    rays (their closest hits from the reference's own trace_world, each bounce ray on the PCG
    stream of its index, as the device generator uses)."""
    cam_idx = random_indices(n_each, per_half, seed)
    camera = pt.camera_rays_at(cam, WIDTH, HEIGHT, 1, cam_idx)
    bounce_idx = random_indices(n_each, per_half, seed + 1)
    prim = pt.camera_rays_at(cam, WIDTH, HEIGHT, 1, bounce_idx)
    res, _ = ref.trace_world(scene, prim)
    hits = np.zeros(len(prim), pt.HIT)
    m = res["hit"] == 1
    hits["t"][m] = res["rec"]["t"][m]
    hits["primitive_id"] = np.where(m, res["rec"]["primitive_id"], -1)
    hits["primitive_type"] = np.where(m, res["rec"]["primitive_type"], 0)
    bounce = pt.bounce_rays_at(scene, prim, hits, 2, bounce_idx)
    return np.concatenate([camera, bounce])


def headline_config(scene, world: int, log2_rays: int = LOG2_RAYS) -> dict:
    """The workload description both arms print (the reference arm times a sample of it)."""
    return {"workload": WORKLOAD, "rays_per_step": 1 << log2_rays, "triangles": int(len(scene.triangles)),
            "bvh_nodes": int(len(scene.nodes)), "image": f"{WIDTH}x{HEIGHT}", "l2": "inputs larger than L2 (940 MB rays)",
            "parallelism": f"replicas x{world}"}


def cpu_reference_rate(scene, rays, ref, threads: int, chunk: int = 1 << 20):
    """Reference trace_world over `rays` on `threads` host threads, in chunks (bounded memory):
    (rays/s, seconds, per-ray mean box tests, per-ray mean primitive tests)."""
    boxes = prims = 0.0
    t = time.perf_counter()
    for b in range(0, len(rays), chunk):
        _, stats = ref.trace_world(scene, rays[b:b + chunk], nthreads=threads)
        boxes += float(stats["boxes"].sum())
        prims += float(stats["primitives"].sum())
    dt = time.perf_counter() - t
    return len(rays) / dt, dt, boxes / len(rays), prims / len(rays)


def run_reference(args):
    """The reference arm: the reference's own trace_world on all host threads, each step a seeded
    random sample of 2^19 of the benchmark's rays (half camera rays, half bounce rays)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_bind import RefCpu
    ref = RefCpu()
    threads = os.cpu_count() or 1
    scene, cam, _ = build_scene()
    per = 1 << 18
    sample = reference_sample(scene, cam, per, ref, seed=11)
    for _ in range(args.warmup):
        cpu_reference_rate(scene, sample, ref, threads)
    t = time.perf_counter()
    for _ in range(args.steps):
        cpu_reference_rate(scene, sample, ref, threads)
    dt = time.perf_counter() - t
    value = len(sample) * args.steps / dt / 1e9
    desc = (f"{len(sample)} rays per step: {per} camera rays and the bounce rays of {per} other camera rays, "
            "at seeded random indices of the 2^24 + 2^24 benchmark rays")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": headline_config(scene, args.gpus), "sample": desc,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": desc + "; trace_world on host_view"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------- rank plumbing
class Ranks:
    """One process per GPU, launched by torchrun: rank, world size, a barrier and the maximum over
    ranks of a measured time.  The closest-hit workload shards as independent replicas (each rank
    walks its own batch; nothing is exchanged on the data path), so the only collectives are the
    barrier around the timed region and the max of the ranks' times.  backend "nccl" keeps the
    reduction on the GPU; "gloo" on the host serves the multi-process tests."""

    def __init__(self, backend: str = "nccl", timeout_s: int = 300):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = torch.device("cuda", self.local) if backend == "nccl" else torch.device("cpu")
        if self.world > 1 and not dist.is_initialized():
            from datetime import timedelta
            extra = {"device_id": self.device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **extra)

    def barrier(self) -> None:
        if self.world > 1:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([x], device=self.device, dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.world > 1 and self.dist.is_initialized():
            self.dist.destroy_process_group()


def whole_job_rate(world: int, units_per_rank: int, steps: int, max_seconds: float) -> float:
    """Units all ranks processed per second of the slowest rank (weak scaling: every rank does
    units_per_rank per step)."""
    return world * units_per_rank * steps / max_seconds


def walk_launches_per_query(ordered: bool) -> int:
    """Kernels one query_device call launches: the walk, plus the ray-key kernel and the sort's
    kernels when the batch is walked in key order (Scene.query_ordered: batches of at least
    2^18 rays on scenes whose walked arrays exceed the L2, under the default setting)."""
    return 1 + (1 + SORT_LAUNCHES if ordered else 0)


# --------------------------------------------------------------------------------------- parity
def _gather(dev_u8, idx, record_bytes, dtype):
    import torch
    return dev_u8.view(-1, record_bytes)[torch.from_numpy(idx.astype(np.int64)).to(dev_u8.device)].cpu().numpy() \
        .view(dtype).reshape(-1)


def closest_parity(scene, rays, hits, oracle, ref, tmax=None, label=""):
    """Our closest hits against the oracle (lowest-id ties, bitwise type / id / t / error) and the
    reference's own trace_world (its last-leaf tie rule: equal wherever no tie decides)."""
    t = time.perf_counter()
    o_hits, ties = oracle.query_ties(scene, rays, tmax=tmax)
    o_s = time.perf_counter() - t
    t = time.perf_counter()
    r_res, r_stats = ref.trace_world(scene, rays, tmax=tmax)
    r_s = time.perf_counter() - t
    same_oracle = ((hits["primitive_type"] == o_hits["primitive_type"]) & (hits["primitive_id"] == o_hits["primitive_id"])
                   & (hits["t"].view(np.uint32) == o_hits["t"].view(np.uint32)) & (hits["error"] == o_hits["error"]))
    r_hit = r_res["hit"] == 1
    r_type = np.where(r_hit, r_res["rec"]["primitive_type"], 0)
    r_id = np.where(r_hit, r_res["rec"]["primitive_id"], -1)
    r_t = np.where(r_hit, r_res["rec"]["t"], 0).astype(np.float32)
    same_ref = (r_type == hits["primitive_type"]) & (r_id == hits["primitive_id"]) & \
               (r_t.view(np.uint32) == hits["t"].view(np.uint32))
    tie = ties > 0
    hit = hits["primitive_type"] != 0
    rel = np.abs(r_t[hit & r_hit] - hits["t"][hit & r_hit]) / np.maximum(np.abs(r_t[hit & r_hit]), 1e-30)
    return {
        "checked": int(len(rays)), "sample": label,
        "mismatches": int((~same_oracle).sum()),
        "reference_mismatches_without_tie": int((~same_ref & ~tie).sum()),
        "ties": int(tie.sum()), "ties_reference_picks_other_id": int((~same_ref & tie).sum()),
        "hits": int(hit.sum()), "errors": int((hits["error"] != 0).sum()),
        "t_max_rel_diff_vs_reference": float(rel.max()) if rel.size else 0.0,
        "oracle_s": o_s, "reference_s": r_s,
        "n_box_reference": float(r_stats["boxes"].mean()), "n_tri_reference": float(r_stats["primitives"].mean()),
        "rule": "type, id, t bitwise vs the oracle (lowest-id ties); vs trace_world wherever no exact-distance tie",
    }


def any_parity(scene, rays, tmax, hits, oracle, ref, label=""):
    """Our any-hit answers against the oracle's any-hit and the reference's trace_world(tmin, tmax).hit."""
    o_hits = oracle.query(scene, rays, mode=pt.QUERY_ANY, tmax=tmax)
    r_res, r_stats = ref.trace_world(scene, rays, tmax=tmax)
    ours = hits["primitive_type"] != 0
    return {"checked": int(len(rays)), "sample": label,
            "mismatches": int((ours != (o_hits["primitive_type"] != 0)).sum()),
            "reference_mismatches": int((ours != (r_res["hit"] == 1)).sum()),
            "occluded": int(ours.sum()), "errors": int((hits["error"] != 0).sum()),
            "n_box_reference": float(r_stats["boxes"].mean()), "n_tri_reference": float(r_stats["primitives"].mean()),
            "rule": "occluded boolean vs the oracle's any-hit and vs trace_world(0.001, tmax).hit"}


# --------------------------------------------------------------------------------------- timing helpers
def timed_queries(dev, rays, n, hits, steps, warmup, tmax=None, mode=pt.QUERY_CLOSEST, ranks=None):
    """warmup + steps query_device calls on the legacy default stream: (step ms total over the
    timed region, max over ranks), walk-kernel ms per launch (events around the walk alone)."""
    import torch
    for _ in range(warmup):
        dev.query_device(rays, n, hits, mode=mode, tmax=tmax)
    torch.cuda.synchronize()
    if ranks:
        ranks.barrier()
    dev.profile(max(1, steps))
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for _ in range(steps):
        dev.query_device(rays, n, hits, mode=mode, tmax=tmax)
    stop.record()
    torch.cuda.synchronize()
    walk = dev.profile_read()
    dev.profile(0)
    total = start.elapsed_time(stop)
    if ranks:
        ranks.barrier()
        total = ranks.max(total)
    return total, walk


def roofline_record(bytes_per_ray, n, walk_ms, hbm, l2_gbs, traffic, kind, extra=None):
    achieved = bytes_per_ray * n / (walk_ms / 1e3) / 1e9
    r = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
         "peak_kind": kind, "kernel": "query_persistent_kernel (the walk)", "kernel_ms": walk_ms,
         "algorithmic_bytes_per_ray": bytes_per_ray}
    if l2_gbs:
        r["l2"] = {"peak_gbs": l2_gbs, "frac": achieved / l2_gbs,
                   "peak_source": "pt_probe_read_bandwidth over a 32 MB L2-resident buffer (16-byte loads)"}
    if traffic:
        r["dram"] = {"gbs": traffic / (walk_ms / 1e3) / 1e9, "frac_of_hbm": traffic / (walk_ms / 1e3) / 1e9 / hbm,
                     "bytes_per_ray": traffic / n}
    if extra:
        r.update(extra)
    return r


# --------------------------------------------------------------------------------------- baselines
def reference_gpu_record(scene, dev, rays_u8, n, value_grays, compat_rays: int = 1 << 20):
    """The reference's own query_rays kernel on the same device-resident rays (same GPU), and
    pt_query_rays_compat against its cuda_query_rays, bytewise, on a slice of `compat_rays` rays
    (the first half of them from the batch's first half, camera rays; the rest from its second half,
    bounce rays for config 2 and surface rays for config 3)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_bind import RefGpuTiming, RefGpu, REF_TIMING_SO, REF_GPU_SO
    if not REF_TIMING_SO.exists() or not REF_GPU_SO.exists():
        return {"unavailable": "oracle/_ref is not built"}
    ms, _ = RefGpuTiming().query(scene, rays_u8.data_ptr(), n, warmup=1, reps=3)
    import torch
    torch.cuda.synchronize()
    k = min(compat_rays, n) // 2 * 2
    half = n // 2
    host = np.concatenate([rays_u8[:k // 2 * 28].cpu().numpy().view(pt.RAY),
                           rays_u8[half * 28:(half + k // 2) * 28].cpu().numpy().view(pt.RAY)])
    t = time.perf_counter()
    theirs = RefGpu().query(scene, host)
    call_s = time.perf_counter() - t
    ours = dev.query_compat(host)
    a, b = ours.view(np.uint8).reshape(k, -1), theirs.view(np.uint8).reshape(k, -1)
    diff = (a != b).any(axis=1)
    return {"grays_per_s": n / ms / 1e6, "kernel_ms": ms, "rays": n,
            "kind": "reference query_rays kernel (src/cuda/cuda_renderer.cu:111-120, one thread per ray, 256 per "
                    "block), scene uploaded by its device_scene, same rays already on the device, same GPU",
            "speedup": value_grays / (n / ms / 1e6),
            "cuda_query_rays_call_s": call_s,
            "compat": {"rays": k, "records_bitwise_equal": int((~diff).sum()), "records_differing": int(diff.sum()),
                       "check": "pt_query_rays_compat vs the reference's cuda_query_rays: all 56 bytes of trace_result"}}


def bvh_node_record(scene, rays, ref, threads: int, our_hits=None):
    """The reference's pre-CUDA host path (bvh_node over triangle objects, virtual hit()) on a
    random sample of the benchmark's rays, on all host cores."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_bind import RefMesh
    tr = scene.triangles
    vertices = np.stack([tr["v0"], tr["v1"], tr["v2"]], axis=1).astype(np.float32)
    t = time.perf_counter()
    mesh = RefMesh(ref, vertices)
    build_s = time.perf_counter() - t
    try:
        t = time.perf_counter()
        tt = mesh.hits(rays, nthreads=threads)
        dt = time.perf_counter() - t
    finally:
        mesh.close()
    rec = {"value": len(rays) / dt / 1e9, "unit": UNIT, "cores": threads, "kind": "reference",
           "sample": f"{len(rays)} of the parity sample's rays; bvh_node::hit over triangle objects "
                     f"(tests/mesh_validation.cpp:76-81), tree built in {build_s:.1f} s (not timed)",
           "seconds": dt}
    if our_hits is not None:
        ours = np.where(our_hits["primitive_type"] != 0, our_hits["t"], -1.0).astype(np.float32)
        rec["hit_agreement"] = float(np.mean((ours < 0) == (tt < 0)))
        both = (ours >= 0) & (tt >= 0)
        rec["t_within_1e-6_rel"] = float(np.mean(np.abs(ours[both] - tt[both]) <= 1e-6 * np.abs(tt[both]))) if both.any() else None
    return rec


# --------------------------------------------------------------------------------------- config 3
C3_PARAMS = dict(sphere_count=128, box_size=1.0, radius_min=0.03, radius_max=0.08, floor=0, light_fraction=0.0,
                 random_triangles=1 << 20, seed=3)
C3_SIDE = 4096


def c3_record(args, hbm, l2_gbs, kind, check_rays: int = 1 << 16):
    """Config 3: 128 displaced spheres of 65,536 triangles + 1,048,576 random triangles (edges
    1e-3..1e-2) in a unit cube under a host SAH tree; 2^25 rays = 2^24 pinhole camera rays (one per
    pixel of 4096x4096) + 2^24 rays leaving random surface points in cosine directions, closest
    hit (tmin 0.001, tmax FLT_MAX); any hit on 2^25 shadow rays between random surface points
    (tmax = distance - 0.001).  Parity on seeded random subsets."""
    import torch
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_bind import Oracle, RefCpu
    t = time.perf_counter()
    scene, cam = pt.procedural_scene(C3_SIDE, C3_SIDE, **C3_PARAMS)
    build_s = time.perf_counter() - t
    dev = pt.Scene(scene)
    n_each = 1 << (args.c3_log2_rays - 1)
    n = 2 * n_each
    rays = torch.empty(n * 28, dtype=torch.uint8, device="cuda")
    hits = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    st = torch.empty(n * 8, dtype=torch.uint8, device="cuda")
    pt.camera_rays_device(cam, C3_SIDE, C3_SIDE, 3, 0, n_each, rays)
    dev.surface_rays_device(4, 0, n_each, rays[n_each * 28:])
    steps, warm = max(3, args.steps // 2), max(3, args.warmup)
    out = {"triangles": int(len(scene.triangles)), "bvh_nodes": int(len(scene.nodes)), "bvh_depth": int(scene.max_depth),
           "scene_build_s": build_s, "device_bytes": dev.device_bytes(), "rays_per_step": n,
           "rays": "2^24 pinhole camera rays (4096x4096, one per pixel) + 2^24 cosine rays from random surface points",
           "l2": "scene (1.5 GB of nodes and triangle records) and rays larger than L2"}
    oracle, ref = Oracle(), RefCpu()
    # closest hit
    total, walk = timed_queries(dev, rays, n, hits, steps, warm)
    dev.query_device(rays, n, hits, stats=st)
    torch.cuda.synchronize()
    stats = st.view(torch.int32).view(-1, 2).to(torch.float64).mean(0).tolist()
    idx = random_indices(n, check_rays, 21)
    par = closest_parity(scene, _gather(rays, idx, 28, pt.RAY), _gather(hits, idx, 16, pt.HIT), oracle, ref,
                         label=f"{len(idx)} seeded random rays of the 2^25")
    b_ray = 32 + 8 + 32 * par["n_box_reference"] + 48 * par["n_tri_reference"]
    b_own = 32 + 8 + 32 * stats[0] + 48 * stats[1]
    walk_ms = float(np.mean(walk))
    out["closest"] = {"value": n * steps / (total / 1e3) / 1e9, "unit": UNIT, "steps": steps, "ms_per_step": total / steps,
                      "kernel_ms": walk_ms, "per_ray": {"child_boxes": stats[0], "primitives": stats[1]},
                      "hit_rate": float((hits.view(torch.int32).view(-1, 4)[:, 2] != 0).float().mean().item()),
                      "gpu_launches": steps * walk_launches_per_query(dev.query_ordered(n)), "parity": par,
                      "roofline": roofline_record(b_ray, n, walk_ms, hbm, l2_gbs,
                                                  profile_summary("query_microbenchmark_ncu.json").get("bytes_per_launch_2^25")
                                                  if n == 1 << 25 else None, kind,
                                                  {"n_box": par["n_box_reference"], "n_tri": par["n_tri_reference"],
                                                   "count_source": "the reference's trace_world on the parity sample",
                                                   "own_counts": {"bytes_per_ray": b_own,
                                                                  "frac": b_own * n / (walk_ms / 1e3) / 1e9 / hbm,
                                                                  "note": "the same formula on this kernel's own box and "
                                                                          "primitive counts; the reference's depth-first walk "
                                                                          "tests about twice as many boxes, which is why the "
                                                                          "fraction above can exceed 1"}})}
    # the reference's own query kernel on the same rays (and its cuda_query_rays on a slice)
    out["closest"]["reference_gpu"] = guarded("c3 reference_gpu", reference_gpu_record, scene, dev, rays, n,
                                              out["closest"]["value"], compat_rays=1 << 18)
    # any hit: shadow rays between surface points
    tmax = torch.empty(n * 4, dtype=torch.uint8, device="cuda")
    dev.surface_rays_device(5, 0, n, rays, tmax=tmax)
    total, walk = timed_queries(dev, rays, n, hits, steps, warm, tmax=tmax, mode=pt.QUERY_ANY)
    dev.query_device(rays, n, hits, mode=pt.QUERY_ANY, tmax=tmax, stats=st)
    torch.cuda.synchronize()
    stats = st.view(torch.int32).view(-1, 2).to(torch.float64).mean(0).tolist()
    idx = random_indices(n, check_rays, 22)
    par = any_parity(scene, _gather(rays, idx, 28, pt.RAY), _gather(tmax, idx, 4, np.float32), _gather(hits, idx, 16, pt.HIT),
                     oracle, ref, label=f"{len(idx)} seeded random shadow rays of the 2^25")
    b_ray = 32 + 4 + 8 + 32 * stats[0] + 48 * stats[1]
    walk_ms = float(np.mean(walk))
    out["any"] = {"value": n * steps / (total / 1e3) / 1e9, "unit": UNIT, "steps": steps, "ms_per_step": total / steps,
                  "kernel_ms": walk_ms, "per_ray": {"child_boxes": stats[0], "primitives": stats[1]},
                  "occluded_rate": float((hits.view(torch.int32).view(-1, 4)[:, 2] != 0).float().mean().item()),
                  "rays": "2^25 shadow rays between two random surface points, tmax = distance - 0.001",
                  "gpu_launches": steps * walk_launches_per_query(dev.query_ordered(n)), "parity": par,
                  "roofline": roofline_record(b_ray, n, walk_ms, hbm, l2_gbs, None, kind,
                                              {"n_box": stats[0], "n_tri": stats[1],
                                               "count_source": "this kernel's own counters (the reference has no "
                                                               "any-hit walk: its shadow query is a closest-hit search)"})}
    dev.close()
    del rays, hits, st, tmax
    torch.cuda.empty_cache()
    return out


def run_c3(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    hbm, _, kind = measured_peaks()
    l2 = pt.read_bandwidth(32 << 20)
    clocks = Clocks(local)
    rec = c3_record(args, hbm, l2, kind)
    clock = clocks.stop()
    c = rec["closest"]
    line = {"metric": "Grays/s closest-hit (traversal microbenchmark)", "value": c["value"], "unit": UNIT, "n_gpus": 1,
            "steps": c["steps"], "warmup": max(3, args.warmup), "ms_per_step": c["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "9.4M-triangle traversal microbenchmark, 2^25 rays", "l2": rec["l2"]},
            "roofline": c["roofline"], "gpu_launches": c["gpu_launches"] + rec["any"]["gpu_launches"], "c3": rec,
            "clocks": clock}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------- batch / mlp
def batch_jobs(count: int, gpu_bvh: bool = False):
    """Seeded render jobs 1..count: log-uniform 10k-2M triangles and 256x256-1920x1080 pixels,
    8-64 spp, bounce limit 4-12, scenes in the style of the procedural 1M-triangle scene."""
    scenes, jobs = [], []
    for i in range(1, count + 1):
        g = np.random.default_rng(1000 + i)
        tris = float(np.exp(g.uniform(np.log(1e4), np.log(2e6))))
        area = float(np.exp(g.uniform(np.log(256 * 256), np.log(1920 * 1080))))
        aspect = float(g.choice([1.0, 4.0 / 3.0, 16.0 / 9.0]))
        w = int(min(1920, max(256, round(np.sqrt(area * aspect)))))
        h = int(min(1080, max(256, round(area / w))))
        spheres = int(min(30, max(1, round(tris / 65536))))
        seg = int(max(8, round(np.sqrt(tris / spheres))))
        scene, cam = pt.procedural_scene(w, h, sphere_count=spheres, segments=seg, rings=max(3, seg // 2 + 1), seed=i,
                                         gpu_bvh=int(gpu_bvh))
        scenes.append(scene)
        jobs.append(dict(scene=i - 1, camera=cam, width=w, height=h, samples=int(g.integers(8, 65)),
                         max_depth=int(g.integers(4, 13)), seed=i))
    return scenes, jobs


def run_batch(args):
    """48 jobs in one graph-captured launch (after a probe autotune); prints one JSON line."""
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    t = time.perf_counter()
    scenes, jobs = batch_jobs(args.jobs, gpu_bvh=args.bvh == "lbvh")
    build_s = time.perf_counter() - t
    b = pt.Batch(scenes, jobs)
    best = b.autotune(probe_samples=1, cache_path=None)
    for _ in range(max(1, args.warmup // 3)):
        b.run()
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    b.run()
    clock = clocks.stop()
    ms, rays, done = b.stats()
    line = {"metric": "Mrays/s batched render", "value": rays / ms / 1e3, "unit": "Mrays/s", "n_gpus": 1, "steps": 1,
            "warmup": max(1, args.warmup // 3), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{len(jobs)} render jobs in one graph launch", "jobs": len(jobs),
                       "triangles": int(sum(len(s.triangles) for s in scenes)),
                       "pixels": int(sum(j["width"] * j["height"] for j in jobs)),
                       "samples": int(sum(j["width"] * j["height"] * j["samples"] for j in jobs)),
                       "autotuned": {"path_capacity": best[0], "block": best[1], "min_active": best[2], "graph": best[3],
                                     "node_width": best[4] if len(best) > 4 else None}},
            "rays": rays, "job_completion_ms": [round(float(x), 3) for x in done], "scene_build_s": build_s,
            "bvh": args.bvh,
            "clocks": clock}
    print(json.dumps(line), flush=True)


def mlp_timings(net, n_query: int = 1 << 21, n_train: int = 1 << 16, reps: int = 20):
    """CUDA-event times of the radiance-cache network alone: a forward pass over n_query
    queries and one Adam step (forward + backward in one launch, then the reduction with the
    update in a second) over n_train samples,
    on seeded synthetic queries in a 10-unit box."""
    import torch
    q = torch.zeros((n_query, 13), dtype=torch.float32, device="cuda")
    g = torch.Generator(device="cuda").manual_seed(5)
    q[:, 0:3] = torch.rand(n_query, 3, device="cuda", generator=g) * 10
    q[:, 3:6] = torch.nn.functional.normalize(torch.randn(n_query, 3, device="cuda", generator=g), dim=1)
    q[:, 6:9] = torch.nn.functional.normalize(torch.randn(n_query, 3, device="cuda", generator=g), dim=1)
    q[:, 9:12] = 0.5
    q[:, 12] = 1.0
    out = torch.zeros(n_query * 3, device="cuda")
    tgt = torch.rand(n_query * 3, device="cuda", generator=g)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps
    fwd_ms = timed(lambda: net.query(q, n_query, out))
    train_ms = timed(lambda: net.train(q, tgt, n_train, wait=False))
    _, tpeak, kind = measured_peaks()
    fwd_tf = 41344.0 * n_query / (fwd_ms / 1e3) / 1e12
    train_tf = 3 * 41344.0 * n_train / (train_ms / 1e3) / 1e12
    return {"forward_queries": n_query, "forward_ms": fwd_ms, "forward_tflops": fwd_tf, "train_samples": n_train,
            "train_step_ms": train_ms, "train_tflops": train_tf, "flop_per_query": 41344,
            "flop_per_training_sample": 3 * 41344, "peak_tflops": tpeak,
            "peak_kind": kind, "launches_per_rep": {"forward": 1, "train": 2}}


def run_mlp(args):
    """The radiance-cache network alone: forward over 2^21 queries, Adam steps over 2^16 samples."""
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    net = pt.RadianceCache((0, 0, 0), (10, 10, 10), seed=1)
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    m = mlp_timings(net, reps=max(1, args.steps))
    clock = clocks.stop()
    line = {"metric": "TFLOP/s radiance-cache MLP forward", "value": m["forward_tflops"], "unit": "TFLOP/s", "n_gpus": 1,
            "steps": max(1, args.steps), "warmup": 3, "ms_per_step": m["forward_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": "MLP 64-64x5-3 forward over 2^21 queries; Adam step over 2^16 samples"},
            "roofline": {"bound": "tensor", "achieved": m["forward_tflops"], "peak": m["peak_tflops"], "unit": "TFLOP/s",
                         "frac": m["forward_tflops"] / m["peak_tflops"], "traffic": None, "peak_kind": m["peak_kind"]},
            "mlp": m, "clocks": clock, "gpu_launches": 3 * (max(1, args.steps) + 3)}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------- config 5
def rel_mse_fn(ref: np.ndarray, var_of_mean: np.ndarray):
    """relMSE = mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2) against the reference r,
    minus the part the reference's own noise contributes (its per-pixel variance of the mean)."""
    denom = ref * ref + 1e-2
    noise = float(np.mean(var_of_mean / denom))

    def rel(x):
        raw = float(np.mean((x - ref) ** 2 / denom))
        return raw - noise, raw
    return rel, noise


def crossing(curve, target):
    """First time (ms) a (samples, ms, relMSE) curve reaches `target`, interpolated log-log
    between the checkpoints either side; None when it never does."""
    for k, (n, t, e) in enumerate(curve):
        if e <= target:
            if k == 0:
                return t
            n0, t0, e0 = curve[k - 1]
            if e0 <= e or e <= 0:
                return t
            f = np.log(e0 / target) / np.log(e0 / e)
            return float(t0 * (t / t0) ** f)
    return None


def cache_record(args, diffuse_only=True, cpu=True):
    """Radiance cache vs plain path tracing on the procedural 1M-triangle scene at 1920x1080,
    depth 12, MIS: relMSE-vs-time curves against an FP64-accumulated plain reference, the time
    each method needs to reach the plain method's 1024-spp relMSE and relMSE <= 1e-3, in wall time
    (host clock around the render calls, the measure the target is stated in) and device time (CUDA events)."""
    W, H, D = 1920, 1080, 12
    t = time.perf_counter()
    scene, cam = pt.procedural_scene(W, H)
    dev = pt.Scene(scene)
    build_s = time.perf_counter() - t
    # reference: plain renders of 256 spp with independent seeds, accumulated in float64
    chunks = max(2, args.ref_spp // 256)
    acc = np.zeros(W * H * 3)
    acc2 = np.zeros(W * H * 3)
    t = time.perf_counter()
    for k in range(chunks):
        r = pt.CudaRenderer(dev, cam, W, H, 100000 + k, max_depth=D)
        r.add_samples(256)
        m = r.sums().astype(np.float64) / 256
        acc += m
        acc2 += m * m
        r.close()
    ref = acc / chunks
    var_of_mean = np.maximum(acc2 / chunks - ref * ref, 0) / (chunks - 1)
    ref_s = time.perf_counter() - t
    del acc, acc2
    rel, noise = rel_mse_fn(ref, var_of_mean)
    plain_marks = sorted({int(round(8 * 1.25 ** k)) for k in range(60) if 8 * 1.25 ** k <= args.max_spp} | {1024})
    # plain path tracer: the progressive renderer
    plain = pt.CudaRenderer(dev, cam, W, H, 1, max_depth=D)
    plain.add_samples(4)                       # warm-up (not counted)
    plain.close()
    plain = pt.CudaRenderer(dev, cam, W, H, 1, max_depth=D)
    plain_curve, wall, done = [], 0.0, 0
    for m in plain_marks:
        t = time.perf_counter()
        plain.add_samples(m - done)
        wall += time.perf_counter() - t
        done = m
        e, _ = rel(plain.sums().astype(np.float64) / m)
        plain_curve.append((m, plain.kernel_milliseconds(), e, wall * 1e3))
        if e <= 1e-3 and m >= 1024:
            break
    plain_rays = plain.rays_traced()
    plain_1024 = next(c for c in plain_curve if c[0] == 1024)
    # radiance cache (library defaults), 32 training-only frames first (counted in its wall time)
    cache = pt.CachedRenderer(dev, cam, W, H, 1, D)
    spf = cache.params.samples_per_frame
    t = time.perf_counter()
    cache.train(32)
    wall = time.perf_counter() - t
    pre_ms = cache.stats()["kernel_ms"]
    cache_curve = []
    for m in plain_marks:
        frames = max(0, -(-m // spf) - cache.stats()["frames"] // spf)
        if frames:
            t = time.perf_counter()
            cache.frames(frames)
            wall += time.perf_counter() - t
        st = cache.stats()
        e, _ = rel(cache.sums().astype(np.float64).reshape(-1) / st["frames"])
        cache_curve.append((st["frames"], st["kernel_ms"], e, wall * 1e3))
        if e <= 1e-3 and st["kernel_ms"] > plain_1024[1]:
            break
    st = cache.stats()
    spec_curve = []
    if diffuse_only:
        spec = pt.CachedRenderer(dev, cam, W, H, 1, D, query_specular=0, spread_threshold=0.01)   # the diffuse-only rule
        spec.train(32)
        for m in (64, 256, 1024):
            spec.frames(max(1, (m - spec.stats()["frames"]) // spf))
            s2 = spec.stats()
            spec_curve.append((s2["frames"], s2["kernel_ms"], rel(spec.sums().astype(np.float64).reshape(-1) / s2["frames"])[0]))
        spec.close()

    def pick(curve, target):
        dev_ms = crossing([(c[0], c[1], c[2]) for c in curve], target)
        wall_ms = crossing([(c[0], c[3], c[2]) for c in curve], target)
        return dev_ms, wall_ms

    c_1e3, c_1e3_wall = pick(cache_curve, 1e-3)
    p_1e3, p_1e3_wall = pick(plain_curve, 1e-3)
    c_1024, c_1024_wall = pick(cache_curve, plain_1024[2])
    eq = min(cache_curve, key=lambda c: abs(c[1] - plain_1024[1]))
    mlp = mlp_timings(cache.cache())
    cache.close()
    plain.close()
    dev.close()
    ratio = lambda a, b: (a / b) if (a and b) else None
    cpu_rec = None
    if cpu:
        sys.path.insert(0, str(ROOT / "oracle"))
        from oracle_bind import RefCpu, REF_CPU_SO
        if REF_CPU_SO.exists() and p_1e3 is not None:
            ref_cpu = RefCpu()
            threads = os.cpu_count() or 1
            small, small_cam = pt.procedural_scene(960, 540)
            t = time.perf_counter()
            _, _, rays = ref_cpu.render(small, small_cam, 960, 540, 1, [2], nthreads=threads)
            dt = time.perf_counter() - t
            rays_to_target = plain_rays / plain_curve[-1][0] * (p_1e3 / plain_curve[-1][1] * plain_curve[-1][0])
            cpu_rec = {"value": rays_to_target / (rays / dt) * 1e3, "unit": "ms", "cores": threads, "kind": "reference",
                       "sample": f"reference trace_pixel_sample (depth 50) on 960x540 x 2 spp: {rays} rays in {dt:.2f} s "
                                 f"= {rays / dt / 1e6:.1f} Mrays/s; value = plain rays to relMSE 1e-3 at that rate"}
    return {
        "workload": "radiance cache vs plain, procedural 1M-triangle scene, 1920x1080, depth 12, MIS",
        "target": "the plain method's 1024-spp relMSE, reached in >= 4x less wall time (the stated target); "
                  "relMSE <= 1e-3 reported beside it",
        "wall_ms": {"cache_to_plain_1024": c_1024_wall, "plain_1024": plain_1024[3], "cache_to_1e-3": c_1e3_wall,
                    "plain_to_1e-3": p_1e3_wall},
        "speedup_wall": {"to_plain_1024": ratio(plain_1024[3], c_1024_wall), "to_1e-3": ratio(p_1e3_wall, c_1e3_wall)},
        "device_ms": {"cache_to_plain_1024": c_1024, "plain_1024": plain_1024[1], "cache_to_1e-3": c_1e3,
                      "plain_to_1e-3": p_1e3, "cache_pretraining": pre_ms},
        "speedup_device": {"to_plain_1024": ratio(plain_1024[1], c_1024), "to_1e-3": ratio(p_1e3, c_1e3)},
        "plain_1024spp_relmse": plain_1024[2],
        "equal_time": {"ms": eq[1], "cache_relmse": eq[2], "plain_relmse_at_1024spp": plain_1024[2]},
        "wall_includes": "cache: its 32 training-only frames, then every frame's render call; plain: every add_samples "
                         "call; both exclude the relMSE evaluation between checkpoints",
        "curves": {"plain": [[c[0], round(c[1], 2), c[2], round(c[3], 2)] for c in plain_curve],
                   "cache": [[c[0], round(c[1], 2), c[2], round(c[3], 2)] for c in cache_curve],
                   "cache_diffuse_only_c0.01": [[c[0], round(c[1], 2), c[2]] for c in spec_curve]},
        "curve_columns": ["samples per pixel", "device ms", "relMSE", "wall ms"],
        "reference": {"spp": chunks * 256, "noise_relmse": noise, "seconds": ref_s},
        "cache_params": {k: getattr(cache.params, k) for k, _ in pt.CachedParams._fields_},
        "cache_stats": st, "mlp": mlp, "scene_build_s": build_s, "cpu_baseline": cpu_rec,
        # per frame: start, the wavefront loop (7 kernels per pair, pairs counted on the device are
        # not read back; 8 pairs is the typical count at 4 samples per frame), the fused tail,
        # forward, resolve, targets, 3 per Adam step (gradients, reduce, update), frame end
        "gpu_launches": int((st["frames"] // spf + 32) * (1 + 7 * 8 + 1 + 3 + 3 * 1 + 1)),
    }


def run_cache(args):
    """The cache_c5 record as its own line (or, with --ref-spp 0, the cost of cached frames)."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    W, H, D = 1920, 1080, 12
    if args.ref_spp <= 0:
        scene, cam = pt.procedural_scene(W, H)
        dev = pt.Scene(scene)
        cache = pt.CachedRenderer(dev, cam, W, H, 1, D, use_graph=0 if args.no_graph else 1)
        cache.train(max(1, args.warmup))
        cache.frames(max(1, args.warmup))
        a = cache.stats()
        clocks = Clocks(local)
        cache.frames(max(1, args.steps))
        clock = clocks.stop()
        b = cache.stats()
        spf = cache.params.samples_per_frame
        ms = b["kernel_ms"] - a["kernel_ms"]
        line = {"metric": "ms per cached frame at 1080p", "value": ms / max(1, args.steps), "unit": "ms", "n_gpus": 1,
                "steps": max(1, args.steps), "warmup": max(1, args.warmup), "ms_per_step": ms / max(1, args.steps),
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32", "data": "synthetic",
                "config": {"workload": "radiance-cache frames, procedural 1M-triangle scene, 1920x1080, depth 12",
                           "samples_per_frame": spf, "graph": not args.no_graph},
                "mrays_per_s": (b["rays"] - a["rays"]) / ms / 1e3,
                "queries_per_frame": (b["queries"] - a["queries"]) / max(1, args.steps),
                "samples_per_frame_trained": (b["samples"] - a["samples"]) / max(1, args.steps), "clocks": clock}
        print(json.dumps(line), flush=True)
        return
    clocks = Clocks(local)
    rec = cache_record(args)
    clock = clocks.stop()
    mlp = rec["mlp"]
    line = {"metric": "ms to the plain method's 1024-spp relMSE at 1080p (radiance cache, wall time)",
            "value": rec["wall_ms"]["cache_to_plain_1024"], "unit": "ms", "n_gpus": 1,
            "steps": rec["cache_stats"]["frames"], "warmup": 32, "ms_per_step": None, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32", "data": "synthetic",
            "config": {"workload": rec["workload"], "l2": "frame state > L2"},
            "roofline": {"bound": "tensor", "kernel": "mlp forward", "achieved": mlp["forward_tflops"], "peak": mlp["peak_tflops"],
                         "unit": "TFLOP/s", "frac": mlp["forward_tflops"] / mlp["peak_tflops"], "traffic": None,
                         "peak_kind": mlp["peak_kind"]},
            "cache_c5": rec, "clocks": clock, "gpu_launches": rec["gpu_launches"],
            "e2e": {"value": rec["wall_ms"]["cache_to_plain_1024"], "unit": "ms", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": W * H * 12, "api": "pt_cached_frames + pt_cached_get_sums (host wall clock)"},
            "cpu_baseline": rec["cpu_baseline"]}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------- config 2 render
def render_record(args, dev=None, scene=None, cam=None, steps: int = 3, warmup: int = 1, cpu: bool = False,
                  W: int = 960, H: int = 600, SPP: int = 64, D: int = 8,
                  workload: str = "progressive render of the procedural 1M-triangle scene, 960x600, 64 spp, bounce limit 8, MIS"):
    """The progressive renderer (one step = a full render from a reset; by default the procedural
    1M-triangle scene, 960x600, 64 spp, bounce limit 8, MIS) beside the reference's own CUDA
    renderer built with its bounce limit set to D ("patched reference", oracle/_ref; D = 50 is the
    reference's own limit, its unpatched build) on the same
    GPU: Mrays/s = rays traced / kernel time, as the reference reports it
    (src/cuda/cuda_renderer.cu:196-213, 246-247), and the two images compared bitwise."""
    t = time.perf_counter()
    if dev is None:
        scene, cam = pt.procedural_scene(W, H)
        dev = pt.Scene(scene)
    build_s = time.perf_counter() - t
    r = pt.CudaRenderer(dev, cam, W, H, 1, max_depth=D)
    for _ in range(max(1, warmup)):
        r.reset(cam)
        r.add_samples(SPP)
    ms = rays = wall = 0.0
    img = None
    for _ in range(steps):
        r.reset(cam)
        t = time.perf_counter()
        r.add_samples(SPP)
        img = r.image()
        wall += time.perf_counter() - t
        ms += r.kernel_milliseconds()
        rays += r.rays_traced()
    r.close()
    value = rays / ms / 1e3
    ref_line = None
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_bind import RefGpu, ref_gpu_so, RefCpu, REF_CPU_SO
    unpatched = D == 50                        # the reference's own bounce limit: its stock build
    if ref_gpu_so(None if unpatched else D).exists():
        gpu = RefGpu(None if unpatched else D)
        rr = gpu.renderer(scene, cam, W, H, 1, mis=True)
        rr.add_samples(SPP)                    # warm-up render
        rr.close()
        rms = rrays = 0.0
        same = True
        for _ in range(steps):
            rr = gpu.renderer(scene, cam, W, H, 1, mis=True)
            rr.add_samples(SPP)
            _, kms, kr = rr.stats()
            rms += kms
            rrays += kr
            same = same and rr.image().tobytes() == img.tobytes()
            rr.close()
        ref_line = {"mrays_per_s": rrays / rms / 1e3, "ms_per_render": rms / steps,
                    "kind": ("reference cuda_renderer, unpatched (its own bounce limit 50), same GPU" if unpatched else
                             f"reference cuda_renderer, bounce limit {D} (patched reference), same GPU"),
                    "images_bit_identical": bool(same), "rays_equal": bool(rrays == rays),
                    "speedup": value / (rrays / rms / 1e3)}
    cpu_rec = None
    if cpu and REF_CPU_SO.exists():
        threads = os.cpu_count() or 1
        t = time.perf_counter()
        _, _, crays = RefCpu().render(scene, cam, W, H, 1, [SPP], nthreads=threads)
        dt = time.perf_counter() - t
        cpu_rec = {"value": crays / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "reference",
                   "sample": f"reference trace_pixel_sample (bounce limit 50) on the same scene, {W}x{H} x {SPP} spp: "
                             f"{crays} rays in {dt:.2f} s"}
    return {"workload": workload,
            "mrays_per_s": value, "ms_per_render": ms / steps, "rays_per_render": rays / steps, "steps": steps,
            "reference_gpu": ref_line, "target": ">= 3x the reference renderer's Mrays/s with identical images" if W == 960 else None,
            "e2e_mrays_per_s": rays / wall / 1e6, "scene_build_s": build_s, "cpu_baseline": cpu_rec}


def run_render(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    clocks = Clocks(local)
    if args.render_scene == "cornell":
        cornell, ccam = pt.cornell_box(320, 200)
        rec = render_record(args, dev=pt.Scene(cornell), scene=cornell, cam=ccam, steps=max(1, args.steps),
                            warmup=max(1, args.warmup), W=320, H=200, SPP=16, D=8, cpu=not args.no_cpu_baseline,
                            workload="Cornell box (20 triangles, 3 spheres), 320x200, 16 spp, bounce limit 8, MIS, seed 1")
        metric = "Mrays/s render (Cornell box, 320x200, 16 spp, depth 8, MIS)"
    else:
        rec = render_record(args, steps=max(1, args.steps), warmup=max(1, args.warmup), cpu=not args.no_cpu_baseline)
        metric = "Mrays/s render (procedural 1M, 960x600, 64 spp, depth 8, MIS)"
    clock = clocks.stop()
    line = {"metric": metric, "value": rec["mrays_per_s"],
            "unit": "Mrays/s", "n_gpus": 1, "steps": rec["steps"], "warmup": max(1, args.warmup),
            "ms_per_step": rec["ms_per_render"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": {"workload": rec["workload"], "l2": "frame state > L2"},
            ("render_c1" if args.render_scene == "cornell" else "render_c2"): rec, "clocks": clock,
            "e2e": {"value": rec["e2e_mrays_per_s"], "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": (320 * 200 if args.render_scene == "cornell" else 960 * 600) * 12,
                    "api": "pt_add_samples + pt_get_image (host wall clock)"},
            "cpu_baseline": rec["cpu_baseline"]}
    print(json.dumps(line), flush=True)


def guarded(name, fn, *a, **k):
    """Runs one sub-record; a failure is recorded in the line instead of ending the run."""
    try:
        return fn(*a, **k)
    except Exception as e:  # noqa: BLE001 - the line reports what failed
        import traceback
        traceback.print_exc()
        return {"error": f"{name}: {type(e).__name__}: {e}"}


# --------------------------------------------------------------------------------------- headline
def main(argv=None):
    args = parse(argv)
    if args.impl == "reference":
        run_reference(args)
        return
    runners = {"batch48": run_batch, "cache": run_cache, "mlp": run_mlp, "render": run_render, "c3": run_c3}
    if args.workload in runners:
        runners[args.workload](args)
        return
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    ranks = Ranks("nccl")
    world, rank, local = ranks.world, ranks.rank, ranks.local
    extras = world == 1 and not args.quick
    hbm, _, peak_kind = measured_peaks()

    scene, cam, t_scene = build_scene()
    t_gpu_build = None
    if args.bvh == "lbvh":
        t = time.perf_counter()
        scene = scene.build_bvh(gpu=True)
        t_gpu_build = time.perf_counter() - t
    dev = pt.Scene(scene)
    n_each = 1 << (args.log2_rays - 1)
    n = 2 * n_each
    rays = torch.empty(n * 28, dtype=torch.uint8, device="cuda")
    hits = torch.empty(n * 16, dtype=torch.uint8, device="cuda")
    pt.camera_rays_device(cam, WIDTH, HEIGHT, 1, 0, n_each, rays)
    dev.query_device(rays, n_each, hits)
    dev.bounce_rays_device(rays, hits, n_each, 2, 0, rays[n_each * 28:])
    torch.cuda.synchronize()

    if args.dump_rays and rank == 0:
        d = Path(args.dump_rays)
        d.mkdir(parents=True, exist_ok=True)
        rays[:n_each * 28].cpu().numpy().tofile(d / "config2_camera_2^24.ray")
        rays[n_each * 28:].cpu().numpy().tofile(d / "config2_bounce_2^24.ray")

    # the timed region: K closest-hit passes over the 2^25 rays (legacy default stream)
    clocks = Clocks(local)
    total_ms, walk = timed_queries(dev, rays, n, hits, args.steps, args.warmup, ranks=ranks)
    clock = clocks.stop()
    walk_ms = float(np.mean(walk))
    value = whole_job_rate(world, n, args.steps, total_ms / 1e3) / 1e9
    hit_rate = float((hits.view(torch.int32).view(-1, 4)[:, 2] != 0).float().mean().item())

    # parity of the timed answers (the hits of the last timed step) on a seeded random subset
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_bind import Oracle, RefCpu, REF_CPU_SO
    parity = None
    have_ref = REF_CPU_SO.exists()
    k_check = args.parity_rays if extras else (1 << 16)
    idx = random_indices(n, k_check, 7)
    sample_rays = _gather(rays, idx, 28, pt.RAY)
    sample_hits = _gather(hits, idx, 16, pt.HIT)
    if have_ref:
        parity = closest_parity(scene, sample_rays, sample_hits, Oracle(), RefCpu(),
                                label=f"{len(idx)} seeded random rays of the 2^25 timed rays (both halves), hits of the "
                                      "last timed step")

    # kernel-own traversal counters (one untimed launch)
    st = torch.empty(n * 8, dtype=torch.uint8, device="cuda")
    dev.query_device(rays, n, hits, stats=st)
    torch.cuda.synchronize()
    stats = st.view(torch.int32).view(-1, 2).to(torch.float64).mean(0).tolist()
    del st

    # end to end through the public host-buffer API: pinned rays in, pinned hits out
    e2e = None
    if not args.no_e2e:
        h_rays = torch.empty(n * 28, dtype=torch.uint8, pin_memory=True)
        h_rays.copy_(rays)
        h_hits = torch.empty(n * 16, dtype=torch.uint8, pin_memory=True)
        lib = pt.library()

        def e2e_step():
            pt.check(lib.pt_query_rays(dev.handle, h_rays.data_ptr(), n, pt.QUERY_CLOSEST, 0.001, None,
                                       h_hits.data_ptr(), None))
        for _ in range(max(1, args.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        ranks.barrier()
        e_steps = max(3, args.steps // 2)
        t = time.perf_counter()
        for _ in range(e_steps):
            e2e_step()
        torch.cuda.synchronize()
        e_dt = ranks.max(time.perf_counter() - t)
        same = bool(h_hits.numpy().tobytes() == hits.cpu().numpy().tobytes())
        e2e = {"value": whole_job_rate(world, n, e_steps, e_dt) / 1e9, "unit": UNIT, "h2d_bytes_per_step": n * 28,
               "d2h_bytes_per_step": n * 16, "ms_per_step": e_dt / e_steps * 1e3,
               "api": "pt_query_rays (host buffers, chunks of 2^20 rays over 3 streams)", "hits_equal_device_path": same}
        del h_rays, h_hits

    # CPU baselines on the host cores (rank 0 at N=1)
    cpu = bvh = None
    threads = os.cpu_count() or 1
    if extras and not args.no_cpu_baseline and have_ref:
        ref = RefCpu()
        # the parity sample repeated until the timed host work reaches ~10 s
        passes, total = 0, 0.0
        while total < 10.0:
            total += cpu_reference_rate(scene, sample_rays, ref, threads)[1]
            passes += 1
        cpu = {"value": passes * len(sample_rays) / total / 1e9, "unit": UNIT, "cores": threads, "kind": "reference",
               "sample": f"the parity sample ({len(sample_rays)} seeded random rays of the 2^25) x {passes} passes, "
                         f"trace_world on host_view, {total:.2f} s"}
        sub = np.arange(0, len(sample_rays), max(1, len(sample_rays) >> 18))
        bvh = guarded("bvh_node", bvh_node_record, scene, sample_rays[sub], ref, threads, sample_hits[sub])

    # roofline of the walk kernel: algorithmic bytes from the reference's own box / primitive counts
    prof = profile_summary()
    traffic = prof.get("bytes_per_launch_2^25")
    l2_gbs = pt.read_bandwidth(32 << 20) if rank == 0 else None
    roofline = None
    if parity:
        n_box, n_tri = parity["n_box_reference"], parity["n_tri_reference"]
        b_ray = 32 + 8 + 32 * n_box + 48 * n_tri
        b_own = 32 + 8 + 32 * stats[0] + 48 * stats[1]
        roofline = roofline_record(b_ray, n, walk_ms, hbm, l2_gbs, traffic, peak_kind,
                                   {"n_box": n_box, "n_tri": n_tri,
                                    "own_counts": {"bytes_per_ray": b_own, "frac": b_own * n / (walk_ms / 1e3) / 1e9 / hbm,
                                                   "n_box": stats[0], "n_tri": stats[1]},
                                    "count_source": "the reference's trace_world on the parity sample (binary tree, "
                                                    "its own visiting order)",
                                    "hbm_read_probe_gbs": pt.read_bandwidth(4 << 30, 4) if rank == 0 else None,
                                    "ncu": prof.get("ncu")})

    ref_gpu = None
    if extras and not args.no_ref_gpu:
        ref_gpu = guarded("reference_gpu", reference_gpu_record, scene, dev, rays, n, value)

    launches = walk_launches_per_query(dev.query_ordered(n))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": headline_config(scene, world, args.log2_rays),
        "kernel_ms": walk_ms, "kernel_stats_per_ray": {"child_boxes": stats[0], "primitives": stats[1]},
        "hit_rate": hit_rate, "scene_build_s": t_scene, "bvh": args.bvh, "gpu_bvh_build_s": t_gpu_build,
        "clocks": clock,
        "gpu_launches": launches * args.steps,
        "gpu_launches_per_step": {"walk": 1, "ray_keys": int(launches > 1), "cub_radix_sort": SORT_LAUNCHES if launches > 1 else 0},
        "parity": parity, "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "cpu_baseline_bvh_node": bvh,
        "reference_gpu": ref_gpu,
    }
    del rays, hits
    torch.cuda.empty_cache()
    if extras and not args.no_render:
        line["render_c2"] = guarded("render_c2", render_record, args, dev=dev, scene=scene, cam=cam)
        line["render_c2_depth50"] = guarded("render_c2_depth50", render_record, args, dev=dev, scene=scene, cam=cam, steps=2, D=50,
                                            workload="progressive render of the procedural 1M-triangle scene, 960x600, 64 spp, "
                                                     "bounce limit 50 (the reference's own), MIS")
        cornell, ccam = pt.cornell_box(320, 200)
        line["render_c1"] = guarded("render_c1", render_record, args, dev=pt.Scene(cornell), scene=cornell, cam=ccam, steps=5,
                                    warmup=2, W=320, H=200, SPP=16, D=8, cpu=True,
                                    workload="Cornell box (20 triangles, 3 spheres), 320x200, 16 spp, bounce limit 8, MIS, seed 1")
    dev.close()
    if extras and not args.no_c3:
        line["c3"] = guarded("c3", c3_record, args, hbm, l2_gbs, peak_kind)
    if extras and not args.no_cache:
        line["cache_c5"] = guarded("cache_c5", cache_record, args, diffuse_only=False, cpu=False)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ranks.close()


if __name__ == "__main__":
    main()
