"""Benchmark: closest-hit rays per second on the procedural 1M-triangle scene.

Workload (one "step"): one closest-hit pass over 2^25 rays of the 1,048,578-triangle procedural
scene (16 displaced spheres of 65,536 triangles, a 2-triangle floor, one emissive quad):
2^24 jittered camera rays of a 960x600 image plus 2^24 cosine-sampled bounce rays leaving their
closest hits, with tmin 0.001 and tmax FLT_MAX as cuda_query_rays uses.  Inputs (940 MB of rays)
are larger than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --workload batch48      48 render jobs of uneven size in one graph launch
  python bench.py --workload cache        radiance cache vs plain path tracing, relMSE vs time at 1080p

--impl reference times the reference's own CPU traversal (trace_world on host_view, built from
its sources into oracle/_ref/) on all host threads over a bounded sample of the same rays.
Under torchrun every rank traces its own replica of the workload (weak scaling, no collective
on the data path); rank 0 prints one JSON line.
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--log2-rays", type=int, default=LOG2_RAYS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", choices=["query", "batch48", "cache", "mlp", "render"], default="query",
                    help="query: the closest-hit benchmark (default); batch48: 48 render jobs in one launch; "
                         "cache: radiance-cache renderer vs plain, time to a relMSE at 1920x1080")
    ap.add_argument("--jobs", type=int, default=48)
    ap.add_argument("--ref-spp", type=int, default=65536,
                    help="cache workload: samples of the FP64 reference image (0: time cached frames only)")
    ap.add_argument("--max-spp", type=int, default=4096, help="cache workload: sample budget of each curve")
    ap.add_argument("--bvh", choices=["sah", "lbvh"], default="sah",
                    help="query and batch48 workloads: the host binned-SAH tree (default) or the linear BVH built on the GPU")
    ap.add_argument("--no-graph", action="store_true",
                    help="cache frames: launch the kernels one by one instead of one graph per frame (for profilers)")
    return ap.parse_args()


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


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


def reference_rays(scene, cam, count_each: int, ref):
    """The first `count_each` camera rays and their bounce rays, built on the host with the
    reference's own trace_world for the camera hits."""
    prim = pt.camera_rays(cam, WIDTH, HEIGHT, 1, 0, count_each)
    res, _ = ref.trace_world(scene, prim)
    hits = np.zeros(count_each, pt.HIT)
    m = res["hit"] == 1
    hits["t"][m] = res["rec"]["t"][m]
    hits["primitive_id"] = np.where(m, res["rec"]["primitive_id"], -1)
    hits["primitive_type"] = np.where(m, res["rec"]["primitive_type"], 0)
    bounce = pt.bounce_rays(scene, prim, hits, 2, 0)
    return np.concatenate([prim, bounce])


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
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_bind import RefCpu
    ref = RefCpu()
    threads = os.cpu_count() or 1
    scene, cam, _ = build_scene()
    per = 1 << 18
    sample = reference_rays(scene, cam, per, ref)
    for _ in range(args.warmup):
        cpu_reference_rate(scene, sample, ref, threads)
    t = time.perf_counter()
    for _ in range(args.steps):
        cpu_reference_rate(scene, sample, ref, threads)
    dt = time.perf_counter() - t
    value = len(sample) * args.steps / dt / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": f"{len(sample)} rays per step (first {per} camera rays + their bounce rays)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{len(sample)} rays per step, trace_world on host_view"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


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
                       "autotuned": {"path_capacity": best[0], "block": best[1], "min_active": best[2], "graph": best[3]}},
            "rays": rays, "job_completion_ms": [round(float(x), 3) for x in done], "scene_build_s": build_s,
            "bvh": args.bvh,
            "clocks": clock}
    print(json.dumps(line), flush=True)


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


def mlp_timings(net, n_query: int = 1 << 21, n_train: int = 1 << 16, reps: int = 20):
    """CUDA-event times of the radiance-cache network alone: a forward pass over n_query
    queries and one Adam step (forward + backward + reduce + update) over n_train samples,
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
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    tpeak = float(peaks.get("bf16_tflops", 1590.0))
    fwd_tf = 41344.0 * n_query / (fwd_ms / 1e3) / 1e12
    train_tf = 3 * 41344.0 * n_train / (train_ms / 1e3) / 1e12
    return {"forward_queries": n_query, "forward_ms": fwd_ms, "forward_tflops": fwd_tf, "train_samples": n_train,
            "train_step_ms": train_ms, "train_tflops": train_tf, "flop_per_query": 41344,
            "flop_per_training_sample": 3 * 41344, "peak_tflops": tpeak,
            "peak_kind": "measured" if peaks else "fallback", "launches_per_rep": {"forward": 1, "train": 3}}


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
            "mlp": m, "clocks": clock, "gpu_launches": 4 * (max(1, args.steps) + 3)}
    print(json.dumps(line), flush=True)


def run_cache(args):
    """Radiance cache vs plain path tracing on the procedural 1M-triangle scene at 1920x1080,
    depth 12, MIS: relMSE-vs-time curves against an FP64-accumulated plain reference, the time
    each method needs to reach relMSE <= 1e-3 and the plain method's 1024-spp relMSE, and
    relMSE at equal time.  Times are device time of the render calls (CUDA events); wall time
    around the same calls is reported beside them."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    W, H, D = 1920, 1080, 12
    t = time.perf_counter()
    scene, cam = pt.procedural_scene(W, H)
    dev = pt.Scene(scene)
    build_s = time.perf_counter() - t
    if args.ref_spp <= 0:
        # frames only (no reference image, no curves): per-frame cost of the cached renderer
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
    clocks = Clocks(local)
    # plain path tracer: the progressive renderer
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
    # radiance cache (library defaults), 32 training-only frames first
    cache = pt.CachedRenderer(dev, cam, W, H, 1, D)
    spf = cache.params.samples_per_frame
    t = time.perf_counter()
    cache.train(32)
    wall = time.perf_counter() - t
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
    clock = clocks.stop()
    st = cache.stats()
    spec = pt.CachedRenderer(dev, cam, W, H, 1, D, query_specular=0, spread_threshold=0.01)   # the diffuse-only rule
    spec.train(32)
    spec_curve = []
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
    tpeak, fwd_tf = mlp["peak_tflops"], mlp["forward_tflops"]
    # CPU baseline: the reference's host renderer's ray rate on a 960x540 render of the same view,
    # turned into the time the plain method's rays to relMSE 1e-3 would take on these cores
    cpu = None
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
        cpu = {"value": rays_to_target / (rays / dt) * 1e3, "unit": "ms", "cores": threads, "kind": "reference",
               "sample": f"reference trace_pixel_sample (depth 50) on 960x540 x 2 spp: {rays} rays in {dt:.2f} s "
                         f"= {rays / dt / 1e6:.1f} Mrays/s; value = plain rays to relMSE 1e-3 at that rate"}
    line = {
        "metric": "ms to relMSE<=1e-3 at 1080p (radiance cache)", "value": c_1e3, "unit": "ms", "n_gpus": 1,
        "steps": st["frames"], "warmup": 32, "ms_per_step": (st["kernel_ms"]) / max(1, st["frames"]),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32", "data": "synthetic",
        "config": {"workload": "radiance cache vs plain, procedural 1M-triangle scene, 1920x1080, depth 12, MIS",
                   "cache": {k: getattr(cache.params, k) for k, _ in pt.CachedParams._fields_},
                   "reference_image": f"{chunks * 256} spp plain, float64 accumulation", "l2": "frame state > L2"},
        "plain_ms_to_1e-3": p_1e3, "speedup_to_1e-3": (p_1e3 / c_1e3) if (p_1e3 and c_1e3) else None,
        "plain_1024spp": {"relmse": plain_1024[2], "ms": plain_1024[1], "cache_ms_to_it": c_1024,
                          "speedup": (plain_1024[1] / c_1024) if c_1024 else None},
        "equal_time": {"ms": eq[1], "cache_relmse": eq[2], "plain_relmse_at_1024spp": plain_1024[2]},
        "wall_ms": {"cache_to_1e-3": c_1e3_wall, "plain_to_1e-3": p_1e3_wall, "cache_to_plain_1024": c_1024_wall},
        "curves": {"plain": [[c[0], round(c[1], 2), c[2]] for c in plain_curve],
                   "cache": [[c[0], round(c[1], 2), c[2]] for c in cache_curve],
                   "cache_diffuse_only_c0.01": [[c[0], round(c[1], 2), c[2]] for c in spec_curve]},
        "reference": {"spp": chunks * 256, "noise_relmse": noise, "seconds": ref_s},
        "cache_stats": st,
        "roofline": {"bound": "tensor", "kernel": "mlp forward", "achieved": fwd_tf, "peak": tpeak, "unit": "TFLOP/s",
                     "frac": fwd_tf / tpeak, "traffic": None, "peak_kind": mlp["peak_kind"]},
        "mlp": mlp,
        "clocks": clock, "scene_build_s": build_s,
        # per frame: start, the wavefront loop (7 kernels per pair, pairs counted on the device
        # are not read back; 8 pairs is the typical count at 4 samples per frame), the fused tail,
        # forward, resolve, targets, 3 per Adam step (gradients, reduce, update), frame end
        "gpu_launches": int((st["frames"] // spf + 32) * (1 + 7 * 8 + 1 + 3 + 3 * cache.params.train_steps + 1)),
        "e2e": {"value": c_1e3_wall, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": W * H * 12,
                "api": "pt_cached_frames + pt_cached_get_sums (host wall clock)"},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_render(args):
    """The progressive renderer on the procedural 1M-triangle scene, 960x600, 64 spp, bounce limit
    8, MIS (one step = a full 64-spp render from a reset), beside the reference's own CUDA
    renderer built with its bounce limit set to 8 ("patched reference", oracle/_ref) on the same
    GPU: Mrays/s = rays traced / kernel time, as the reference reports it, and the two images
    compared bitwise."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    W, H, SPP, D = 960, 600, 64, 8
    t = time.perf_counter()
    scene, cam = pt.procedural_scene(W, H)
    dev = pt.Scene(scene)
    build_s = time.perf_counter() - t
    r = pt.CudaRenderer(dev, cam, W, H, 1, max_depth=D)
    for _ in range(max(1, args.warmup)):
        r.reset(cam)
        r.add_samples(SPP)
    clocks = Clocks(local)
    ms = rays = 0.0
    wall = 0.0
    steps = max(1, args.steps)
    img = None
    for _ in range(steps):
        r.reset(cam)
        t = time.perf_counter()
        r.add_samples(SPP)
        img = r.image()
        wall += time.perf_counter() - t
        ms += r.kernel_milliseconds()
        rays += r.rays_traced()
    clock = clocks.stop()
    value = rays / ms / 1e3
    ref_line = None
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_bind import RefGpu, ref_gpu_so, RefCpu, REF_CPU_SO
    if ref_gpu_so(D).exists():
        gpu = RefGpu(D)
        rr = gpu.renderer(scene, cam, W, H, 1, mis=True)
        rr.add_samples(SPP)                    # warm-up render
        rr.close()
        rms = rrays = 0.0
        for _ in range(steps):
            rr = gpu.renderer(scene, cam, W, H, 1, mis=True)
            rr.add_samples(SPP)
            _, kms, kr = rr.stats()
            rms += kms
            rrays += kr
            same = rr.image().tobytes() == img.tobytes()
            rr.close()
        ref_line = {"mrays_per_s": rrays / rms / 1e3, "ms_per_render": rms / steps,
                    "kind": "reference cuda_renderer, bounce limit 8 (patched reference), same GPU",
                    "images_bit_identical": bool(same), "speedup": value / (rrays / rms / 1e3)}
    cpu = None
    if REF_CPU_SO.exists():
        threads = os.cpu_count() or 1
        t = time.perf_counter()
        _, _, crays = RefCpu().render(scene, cam, W, H, 1, [SPP], nthreads=threads)
        dt = time.perf_counter() - t
        cpu = {"value": crays / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "reference",
               "sample": f"reference trace_pixel_sample (bounce limit 50) on the same scene, {W}x{H} x {SPP} spp: {crays} rays in {dt:.2f} s"}
    line = {"metric": "Mrays/s render (procedural 1M, 960x600, 64 spp, depth 8, MIS)", "value": value, "unit": "Mrays/s",
            "n_gpus": 1, "steps": steps, "warmup": max(1, args.warmup), "ms_per_step": ms / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "progressive render of the procedural 1M-triangle scene, 960x600, 64 spp, bounce limit 8, MIS",
                       "l2": "frame state > L2"},
            "rays_per_render": rays / steps, "reference_gpu": ref_line, "clocks": clock, "scene_build_s": build_s,
            "e2e": {"value": rays / wall / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": W * H * 12,
                    "api": "pt_add_samples + pt_get_image (host wall clock)"},
            "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "batch48":
        run_batch(args)
        return
    if args.workload == "cache":
        run_cache(args)
        return
    if args.workload == "mlp":
        run_mlp(args)
        return
    if args.workload == "render":
        run_render(args)
        return
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    ranks = Ranks("nccl")
    world, rank, local = ranks.world, ranks.rank, ranks.local
    barrier, max_over_ranks = ranks.barrier, ranks.max

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

    stream = 0   # legacy default stream: torch's current stream here, and the library's launches
    launches = []
    for _ in range(args.warmup):
        dev.query_device(rays, n, hits, stream=stream)
    torch.cuda.synchronize()
    barrier()
    clocks = Clocks(local)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    start.record()
    for k in range(args.steps):
        ev[k][0].record()
        dev.query_device(rays, n, hits, stream=stream)
        ev[k][1].record()
    stop.record()
    torch.cuda.synchronize()
    clock = clocks.stop()
    barrier()
    total_ms = max_over_ranks(start.elapsed_time(stop))
    per_launch_ms = [a.elapsed_time(b) for a, b in ev]
    kernel_ms = float(np.mean(per_launch_ms))
    value = whole_job_rate(world, n, args.steps, total_ms / 1e3) / 1e9

    # kernel-own traversal counters (one untimed launch)
    st = torch.empty(n * 8, dtype=torch.uint8, device="cuda")
    dev.query_device(rays, n, hits, stats=st)
    torch.cuda.synchronize()
    stats = st.view(torch.int32).view(-1, 2).to(torch.float64).mean(0).tolist()
    hit_rate = float((hits.view(torch.int32).view(-1, 4)[:, 2] != 0).float().mean().item())

    # end to end through the public host-buffer API: pinned rays in, pinned hits out
    e2e = None
    if not args.no_e2e:
        h_rays = torch.empty(n * 28, dtype=torch.uint8, pin_memory=True)
        h_rays.copy_(rays)
        h_hits = torch.empty(n * 16, dtype=torch.uint8, pin_memory=True)
        r_np = h_rays.numpy().view(pt.RAY)
        lib = pt.library()

        def e2e_step():
            pt.check(lib.pt_query_rays(dev.handle, h_rays.data_ptr(), n, pt.QUERY_CLOSEST, 0.001, None,
                                       h_hits.data_ptr(), None))
        for _ in range(max(1, args.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        barrier()
        e_steps = max(3, args.steps // 2)
        t = time.perf_counter()
        for _ in range(e_steps):
            e2e_step()
        torch.cuda.synchronize()
        e_dt = max_over_ranks(time.perf_counter() - t)
        e2e = {"value": whole_job_rate(world, n, e_steps, e_dt) / 1e9, "unit": UNIT, "h2d_bytes_per_step": n * 28,
               "d2h_bytes_per_step": n * 16, "ms_per_step": e_dt / e_steps * 1e3,
               "api": "pt_query_rays (host buffers, 3-stream chunked pipeline)"}
        assert h_hits.numpy().view(pt.HIT).size == len(r_np)

    # CPU baseline: the reference's own trace_world on the host cores, bounded sample
    cpu = None
    n_box = n_tri = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        from oracle_bind import RefCpu, REF_CPU_SO
        if REF_CPU_SO.exists():
            ref = RefCpu()
            threads = os.cpu_count() or 1
            # grow the sample until it holds ~10 s of traversal on all host cores (cap 2^23 + 2^23 rays)
            per = 1 << 16
            sample = reference_rays(scene, cam, per, ref)
            rate, dt, n_box, n_tri = cpu_reference_rate(scene, sample, ref, threads)
            while dt < 10.0 and per < (1 << 23):
                per = min(1 << 23, per * max(2, 1 << int(np.log2(max(1.0, 10.0 / max(dt, 1e-3))))))
                sample = reference_rays(scene, cam, per, ref)
                rate, dt, n_box, n_tri = cpu_reference_rate(scene, sample, ref, threads)
            # at the cap, repeat the sample until the timed CPU work reaches ~10 s
            passes, total = 1, dt
            while total < 10.0:
                total += cpu_reference_rate(scene, sample, ref, threads)[1]
                passes += 1
            rate = passes * len(sample) / total
            cpu = {"value": rate / 1e9, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"{len(sample)} rays (first {per} camera rays + their bounce rays) x {passes} passes, "
                             f"trace_world on host_view, {total:.2f} s"}

    peak, peak_kind = measured_peaks()
    roofline = None
    if n_box is not None:
        bytes_per_ray = 32 + 8 + 32 * n_box + 48 * n_tri
        achieved = bytes_per_ray * n / (kernel_ms / 1e3) / 1e9
        traffic = None
        prof = ROOT / "profiles" / "traffic.json"
        if prof.exists():
            traffic = json.loads(prof.read_text()).get("query_closest_bytes_per_launch")
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "peak_kind": peak_kind,
                    "algorithmic_bytes_per_ray": bytes_per_ray, "n_box": n_box, "n_tri": n_tri}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "rays_per_step": n, "triangles": int(len(scene.triangles)),
                   "bvh_nodes": int(len(scene.nodes)), "image": f"{WIDTH}x{HEIGHT}", "l2": "inputs larger than L2 (940 MB rays)",
                   "parallelism": f"replicas x{world}"},
        "kernel_ms": kernel_ms, "kernel_stats_per_ray": {"child_boxes": stats[0], "primitives": stats[1]},
        "hit_rate": hit_rate, "scene_build_s": t_scene, "bvh": args.bvh, "gpu_bvh_build_s": t_gpu_build,
        "clocks": clock,
        # per step: the ray-key kernel, the radix sort of the keys (CUB DeviceRadixSort, 30 bits)
        # and the walk kernel; the sort's own kernels are counted as one launch here
        "gpu_launches": 3 * args.steps,
        "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    del dev
    ranks.close()


if __name__ == "__main__":
    main()
