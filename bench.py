"""Benchmark of the B200 std/path backend: paths/s of the plain method, large config.

One step = one animation frame of the large configuration: the frame's 1,000,000
boid-placed instance transforms rebuild the TLAS, then a 1920x1080, 64 spp, depth-8
render (132.7 M paths) runs through the wavefront.  `value` is measured with the
inputs resident in HBM (device rows, device image) by CUDA events on the library's
stream; `e2e` goes through the public C ABI with pinned host rows in and the host
image out, both copies inside the timed region.  Multi-GPU (torchrun): every rank
renders its own frames (weak scaling, no collective on the data path).

At one GPU the same line then carries compact blocks of the other configurations, each
timed with its own clock record: `small` (the 256x256 configuration), `batch` (256
batched preview jobs vs sequential plain renders), `cache` (the learned radiance cache on the frame scene vs plain, with errors
against a 1024-spp plain render and the FP64 oracle) and `serve` (continuous batching
vs the plain path served FIFO on one Poisson trace).  `--config batch|cache|serve` runs
each at full size.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--config large|small|profile|batch|serve|cache] [--no-blocks]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
METRIC = "paths/s and p50/p99 render latency vs plain CUDA path at ≤1% RMSE, 1 B200"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d.get("bf16_tflops", PEAKS_FALLBACK["bf16_tflops"])),
                "source": "measured"}
    return {**PEAKS_FALLBACK, "source": "fallback"}


def workload(config: str, seed: int = 0):
    from vork_b200 import Profile, scene
    if config == "small":
        sc = scene.spheres_scene(seed=seed)
        prof = Profile.reference_transport(4, 16)
        return sc, None, prof, {"workload": "plain-small: 256x256, 16 spp, depth 4, 64 UV spheres + 8192-tri grid, 1 area light"}
    if config == "profile":
        # The large scene (BVH data far larger than L2) at 480x270 and 4 spp: a case small
        # enough for a full ncu capture of one launch.
        sc, flock = scene.flock_scene(seed=seed, width=480, height=270)
        prof = Profile.reference_transport(8, 4)
        return sc, flock, prof, {"workload": "plain-large scene at 480x270, 4 spp, depth 8 (profiling case)"}
    sc, flock = scene.flock_scene(seed=seed)
    prof = Profile.reference_transport(8, 64)
    return sc, flock, prof, {"workload": "plain-large: 1920x1080, 64 spp, depth 8, 1,000,000 boid-placed instances of a 500-tri "
                                         "geodesic mesh (500M instanced tri) + 2M-tri terrain, sun + constant sky, TLAS rebuilt per frame"}


def frames_for(sc, flock, count):
    """Per-frame instance rows (N,12): the flock advanced one step per frame."""
    out = []
    for _ in range(count):
        if flock is None:
            out.append(np.ascontiguousarray(sc.instance_rows, np.float32).reshape(-1, 12))
            continue
        flock.step()
        rows = np.concatenate([flock.rows(), sc.instance_rows[-1:]], 0)
        out.append(np.ascontiguousarray(rows, np.float32).reshape(-1, 12))
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None, "reasons": sorted(reasons),
                "samples": len(sm)}


# Algorithmic bytes of the closest-hit trace per unit of work, fixed independently of the
# node format this backend stores: a node visit is 80 B (one compressed 8-wide node: eight
# quantised child boxes plus header and child references), a triangle test 36 B (three
# fp32 corners), an instance entry 64 B (its TLAS leaf record: world->object rows and BLAS
# references), and a ray 32 B of queue entry read plus a 24 B hit record written.
NODE_BYTES, TRI_BYTES, INSTANCE_BYTES, RAY_BYTES = 80, 36, 64, 32 + 24
# What the 4-wide FP32 node format actually stores and the kernel requests per visit:
# 112 of its 128 bytes (6 face planes x 16 B + four child references), 48 B per stored
# triangle (3 x float4), 20 B per hit record.
STORED_NODE_BYTES, STORED_TRI_BYTES, STORED_RAY_BYTES = 112, 48, 32 + 20


def roofline_bytes(stats: dict) -> float:
    """Algorithmic bytes of the closest-hit trace kernels of one render (node, triangle
    and instance visits counted exactly by the instrumented traversal)."""
    return (stats["nodes_visited"] * NODE_BYTES + stats["triangles_tested"] * TRI_BYTES
            + stats["instances_entered"] * INSTANCE_BYTES + stats["extension_rays"] * RAY_BYTES)


def stored_bytes(stats: dict) -> float:
    """The same visits at the stored sizes of this backend's 4-wide FP32 nodes."""
    return (stats["nodes_visited"] * STORED_NODE_BYTES + stats["triangles_tested"] * STORED_TRI_BYTES
            + stats["instances_entered"] * INSTANCE_BYTES + stats["extension_rays"] * STORED_RAY_BYTES)


def trace_limiter():
    """What ncu shows limits the closest-hit trace (profiles/trace_closest_limiter.json,
    written from the full capture of the profiling case); None when absent."""
    f = ROOT / "profiles" / "trace_closest_limiter.json"
    return json.loads(f.read_text()) if f.exists() else None


def cpu_baseline(config: str, seconds: float = 12.0):
    """The oracle's FP32 restatement of the path (the reference has no CPU path tracer and
    its Vulkan path cannot run here) on the same frame, all host threads: the whole frame
    at one sample per pixel, repeated over sample indices until about `seconds`."""
    from oracle import pyoracle
    from vork_b200 import Profile
    sc, flock, prof, _ = workload(config)
    o = pyoracle.OracleScene(sc, fp32=True, fp64=False)
    cam = sc.camera
    threads = os.cpu_count() or 1
    w, h = cam.width, cam.height
    p = Profile.reference_transport(prof.bounces[0], prof.samples, sample_count=1)
    o.render(p.c(), w // 2 - 4, h // 2 - 4, 8, 8, fp64=False, threads=threads)  # bakes the oracle's BRDF atlas
    spp, dt = 0, 0.0
    while dt < seconds and spp < prof.samples:
        p = Profile.reference_transport(prof.bounces[0], prof.samples, first_sample=spp, sample_count=1)
        t0 = time.perf_counter()
        o.render(p.c(), 0, 0, w, h, fp64=False, threads=threads)
        dt += time.perf_counter() - t0
        spp += 1
    o.close()
    return {"value": w * h * spp / dt, "unit": "paths/s", "cores": threads, "kind": "port",
            "sample": f"whole {w}x{h} frame at {spp} spp (of {prof.samples}, one sample per call), depth {prof.bounces[0]}, "
                      f"FP32 C++ restatement, {threads} threads, {dt:.1f} s"}


def run_reference(args, rank):
    """--impl reference: the reference's path on host cores.  The reference has no CPU
    path tracer and its Vulkan path cannot run on this box, so its C++ restatement (the
    oracle, FP32) stands in.  One step = the whole frame at one sample per pixel (sample
    index = step), the same frame, depth and threads as `cpu_baseline`, so the two agree."""
    if rank != 0:
        return
    from oracle import pyoracle
    from vork_b200 import Profile
    sc, flock, prof, cfg = workload(args.config)
    o = pyoracle.OracleScene(sc, fp32=True, fp64=False)
    cam = sc.camera
    threads = os.cpu_count() or 1
    w, h = cam.width, cam.height

    def step(k):
        p = Profile.reference_transport(prof.bounces[0], prof.samples, first_sample=k % prof.samples, sample_count=1)
        o.render(p.c(), 0, 0, w, h, fp64=False, threads=threads)

    for k in range(args.warmup):
        step(k)
    times = []
    for k in range(args.steps):
        t0 = time.perf_counter()
        step(args.warmup + k)
        times.append(time.perf_counter() - t0)
    o.close()
    total = sum(times)
    value = args.steps * w * h / total
    line = {"metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded generator; no dataset)", "impl": "reference",
            "config": {**cfg, "parallelism": "host cores", "l2_flush": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": "paths/s", "cores": threads, "kind": "port",
                             "sample": f"whole {w}x{h} frame at 1 spp per step (sample index = step), depth {prof.bounces[0]}, "
                                       f"{threads} threads; the reference's Vulkan path cannot run on this box, so its C++ "
                                       "restatement (FP32) stands in"},
            "e2e": {"value": value, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def clocks_ok(summary: dict) -> bool:
    """A timed region is kept only without hardware or thermal slowdown (power capping is
    noted, not rejected)."""
    bad = {"hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"}
    return not (set(summary.get("reasons") or []) & bad)


def small_block(r, frames: int = 400, warmup: int = 5) -> dict:
    """The small configuration (256x256, 16 spp, depth 4, 64 spheres + 8192-triangle grid,
    one area light): device time of whole renders into a device image, and end to end
    with the host image out, over `frames` renders."""
    import torch
    from vork_b200 import Profile, abi, scene
    sc = scene.spheres_scene(seed=0)
    prof = Profile.reference_transport(4, 16)
    cam = sc.camera
    paths = cam.width * cam.height * prof.samples
    with r.install(sc) as s:
        stream = torch.cuda.ExternalStream(r.stream, device=torch.device("cuda", r.device))
        image = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device=f"cuda:{r.device}")
        host = torch.empty((cam.height, cam.width, 4), dtype=torch.float32).pin_memory()
        for _ in range(warmup):
            s.render(prof, device_ptr=image.data_ptr())
        torch.cuda.synchronize()
        with ClockSampler(r.device) as clocks:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            for _ in range(frames):
                s.render(prof, device_ptr=image.data_ptr())
            ev1.record(stream)
            torch.cuda.synchronize()
            dev_ms = ev0.elapsed_time(ev1)
            t0 = time.perf_counter()
            for _ in range(frames):
                s.render(prof, out=host.numpy())
            e2e_s = time.perf_counter() - t0
    return {"workload": "plain-small: 256x256, 16 spp, depth 4, 64 UV spheres + 8192-tri grid, 1 area light",
            "value": frames * paths / (dev_ms / 1000.0), "unit": "paths/s", "ms_per_frame": dev_ms / frames,
            "e2e": {"value": frames * paths / e2e_s, "unit": "paths/s", "d2h_bytes_per_step": int(cam.width * cam.height * 16)},
            "frames": frames, "clocks": clocks.summary()}


def batch_block(r, jobs: int, warmup: int) -> dict:
    """Batched previews: `jobs` seeded jobs in one shared wavefront (graphs replayed per
    wave, wave shape from the autotuner) against one plain render per job in sequence;
    per-job images are bit-identical between the arms (the test suite checks that)."""
    import torch
    from vork_b200 import Profile, abi, scene
    t_block = time.perf_counter()
    items = [(r.install(sc), Profile.reference_transport(depth, spp)) for sc, spp, depth in scene.preview_jobs(jobs, seed=0)]
    paths = sum(i.scene.camera.width * i.scene.camera.height * p.samples for i, p in items)
    tune = r.autotune(items)
    # Host images written in place by both arms, allocated and touched up front (fresh
    # pages would add their first-touch faults to whichever arm writes them first).
    outs = [np.zeros((i.scene.camera.height, i.scene.camera.width, 4), np.float32) for i, _ in items]
    for _ in range(max(1, warmup)):
        r.render_batch(items, outs=outs)
        for (inst, prof), o in zip(items[:8], outs):
            inst.render(prof, out=o)
    torch.cuda.synchronize()
    with ClockSampler(r.device) as clocks:
        t0 = time.perf_counter()
        for (inst, prof), o in zip(items, outs):
            inst.render(prof, out=o)
        seq_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        _, st = r.render_batch(items, outs=outs)
        batch_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        r.render_batch(items, flags=4, outs=outs)  # fair scheduling (one sample of every job per wave)
        fair_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        r.render_batch(items, flags=abi.PROFILE_SERIAL_WAVES, outs=outs)  # waves one after another, graphs replayed
        serial_s = time.perf_counter() - t0
    for inst, _ in items:
        inst.close()
    return {"workload": f"batched previews: {len(items)} jobs, resolution log-uniform 128^2..1024^2, spp U{{4..32}}, depth U{{4..8}}, "
                        "1k-200k-triangle sphere scenes seeded per job; host images out, copies in the timed region",
            "paths": paths, "value": paths / batch_s, "unit": "paths/s", "makespan_ms": 1000 * batch_s,
            "sequential": {"value": paths / seq_s, "unit": "paths/s", "makespan_ms": 1000 * seq_s},
            "fair_schedule": {"value": paths / fair_s, "unit": "paths/s", "makespan_ms": 1000 * fair_s},
            "one_stream": {"value": paths / serial_s, "unit": "paths/s", "makespan_ms": 1000 * serial_s},
            "speedup_vs_sequential": seq_s / batch_s,
            "autotune": {k: tune[k] for k in ("best_capacity", "best_blocks_per_sm", "best_ms")},
            "gpu_launches": st["kernel_launches"], "clocks": clocks.summary(), "block_wall_s": time.perf_counter() - t_block}


def serve_scenes(r, flock_inst=None, flock=None):
    """The serving mix's resident scenes: four from the small configuration's generator
    (1k-200k triangles, log-uniform) and two boid flocks from the large one (20,000 birds
    and, when given, the installed 1,000,000-bird frame scene), with 24 frames of
    instance rows for each flock (its sequences are animated)."""
    from vork_b200 import scene
    rng = np.random.default_rng(0)
    scenes, animations, names = [], {}, []
    for k in range(4):
        tris = float(np.exp(rng.uniform(np.log(1000), np.log(200_000))))
        cells = 8 if tris < 20000 else 64
        n = max(1, int(round((tris - 2 * cells * cells) / 960)))
        scenes.append(r.install(scene.spheres_scene(num_spheres=n, seed=k, grid_cells=cells, width=1920, height=1080)))
        names.append(f"spheres x{n} ({n * 960 + 2 * cells * cells} tri)")
    small, small_flock = scene.flock_scene(num_birds=20_000, seed=5, terrain_cells=200)
    scenes.append(r.install(small))
    names.append("flock 20k birds (10M instanced tri)")
    owned = len(scenes)
    flocks = [(4, small, small_flock)]
    if flock_inst is not None:
        scenes.append(flock_inst)
        names.append("flock 1M birds (500M instanced tri + 2M-tri terrain)")
        flocks.append((5, flock_inst.scene, flock))
    for idx, sc, fl in flocks:
        frames = []
        for _ in range(24):
            fl.step()
            frames.append(np.ascontiguousarray(np.concatenate([fl.rows(), sc.instance_rows[-1:]], 0), np.float32))
        animations[idx] = frames
    return scenes, animations, names, owned


def serve_block(r, requests: int, rates, schedule: str = "srpt", fifo: bool = True, flock_inst=None, flock=None,
                timeout_s: float = 1500.0, wave_slots: int = 0, serial: bool = False) -> dict:
    """Serving: Poisson arrivals at each rate of 80% stills / 20% 24-frame sequences (the
    flocks' sequences animated: TLAS rebuilt per frame through a fork), resolution per
    request log-uniform 256x256..1920x1080, spp U{8..128}, depth 8, 160 GB admission
    budget; continuous batching against the plain path served FIFO on the same trace."""
    import copy
    from vork_b200.serving import Server, fifo_load, poisson_load, request_mix
    t_block = time.perf_counter()
    scenes, animations, names, owned = serve_scenes(r, flock_inst, flock)
    from vork_b200 import abi
    flags = {"srpt": 0, "aged": 0, "fair": 4, "packed": 8}[schedule] | (abi.PROFILE_SERIAL_WAVES if serial else 0)
    aging = 2e8 if schedule == "aged" else 0.0   # paths per second waited: about the device's rate on these scenes
    out = []
    for i, rate in enumerate(rates):
        reqs = request_mix(requests, len(scenes), seed=i, frames=24, spp_range=(8, 128), bounces=8,
                           pixels_range=(256 * 256, 1920 * 1080))
        row = {"rate": rate}
        with ClockSampler(r.device) as clocks:
            with Server(r, memory_budget_bytes=160 << 30, max_jobs=256, flags=flags, aging_paths_per_s=aging,
                        wave_capacity=wave_slots) as srv:
                row["continuous"] = poisson_load(srv, scenes, copy.deepcopy(reqs), rate=rate, seed=i, timeout_s=timeout_s,
                                                 animations=animations)
        row["continuous"]["clocks"] = clocks.summary()
        if fifo:
            with ClockSampler(r.device) as clocks:
                row["fifo_plain"] = fifo_load(scenes, copy.deepcopy(reqs), rate=rate, seed=i, timeout_s=timeout_s, animations=animations)
            row["fifo_plain"]["clocks"] = clocks.summary()
            row["p50_speedup"] = row["fifo_plain"]["p50_s"] / row["continuous"]["p50_s"]
            row["p99_speedup"] = row["fifo_plain"]["p99_s"] / row["continuous"]["p99_s"]
            row["throughput_speedup"] = row["continuous"]["throughput_paths_s"] / row["fifo_plain"]["throughput_paths_s"]
        row["sequences"] = sum(1 for q in reqs if q.frames > 1)
        out.append(row)
    for sc in scenes[:owned]:
        sc.close()
    return {"workload": f"serving: {requests} requests per rate, Poisson rates {list(rates)} req/s, 80% stills / 20% 24-frame "
                        "sequences (flock sequences animated, TLAS rebuilt per frame through a fork), resolution log-uniform "
                        "256x256..1920x1080 per request, spp U{8..128}, depth 8, 160 GB budget, continuous batching "
                        f"({schedule} waves) vs the plain path served FIFO",
            "scenes": names, "rates": out, "block_wall_s": time.perf_counter() - t_block}


def _errors(img, ref, h16):
    blocks = lambda im: im[:h16].reshape(h16 // 16, 16, im.shape[1] // 16, 16, 3).mean((1, 3))
    br = blocks(ref)
    return {"mean_rel_err": float(img.mean() / ref.mean() - 1.0),
            "rel_rmse_pixels": float(np.sqrt(np.mean((img - ref) ** 2)) / ref.mean()),
            "rel_rmse_16x16_blocks": float(np.sqrt(np.mean((blocks(img) - br) ** 2)) / br.mean())}


def cache_block(r, s, sc, frames, warmup: int, steps: int, errors: bool = True, ref_spp: int = 1024, pretrain: int = 16) -> dict:
    """Learned radiance cache on the large scene, 16 spp, depth 8: per frame the TLAS is
    rebuilt, the cache takes one online training round (2^16 records, 4 Adam steps) and
    renders through it (paths stop at vertex 2); against plain 16-spp renders of the same
    frames, after `pretrain` untimed training rounds (earlier frames of the sequence).  Error of both against the plain tracer at `ref_spp` of the last frame, and
    of the 64x64 centre crop against the FP64 oracle."""
    import torch
    from vork_b200 import Profile, RadianceCache, abi
    t_block = time.perf_counter()
    spp, depth = 16, 8
    cam = sc.camera
    npix = cam.width * cam.height
    n_inst = frames[0].shape[0]
    dev_frames = [torch.from_numpy(frames[i % len(frames)]).to(f"cuda:{r.device}") for i in range(warmup + steps)]
    prof = Profile.reference_transport(depth, spp, seed=1)
    timed = prof.__class__(**{**prof.__dict__, "flags": abi.PROFILE_TIME_KERNELS})
    k = RadianceCache(s, seed=0)
    cached_ms, plain_ms, train_ms, build_ms, cache_ms, queries = [], [], [], [], 0.0, 0
    train_parts = {"paths_ms": 0.0, "steps_ms": 0.0, "host_ms": 0.0}
    rays_cached = rays_plain = 0
    # An animated sequence trains the cache every frame; before the measured frames it has
    # seen `pretrain` rounds (untimed), as it would have after that many earlier frames.
    s.update_instances_device(dev_frames[0].data_ptr(), n_inst, 1)
    for i in range(pretrain):
        k.train(Profile.reference_transport(depth, 1, seed=500 + i))
    with ClockSampler(r.device) as clocks:
        for i in range(warmup + steps):
            s.update_instances_device(dev_frames[i].data_ptr(), n_inst, 1)
            b = s.info()["build_ms"]
            t = k.train(Profile.reference_transport(depth, 1, seed=1000 + i))
            c = k.render(timed)
            p = s.render(timed)
            if i >= warmup:
                build_ms.append(b); train_ms.append(t["train_ms"])
                for key in train_parts:
                    train_parts[key] += t[key] / steps
                cached_ms.append(t["train_ms"] + c.stats["render_ms"]); plain_ms.append(p.stats["render_ms"])
                cache_ms += c.stats["cache_ms"]; queries += c.stats["cache_queries"]
                rays_cached += c.stats["extension_rays"]; rays_plain += p.stats["extension_rays"]
    last_cached, last_plain = c.image[..., :3], p.image[..., :3]
    paths = npix * spp * steps
    pk = peaks()
    flops = 2.0 * abi.NRC_MLP_PARAMS * queries
    tflops = flops / (cache_ms / 1000.0) / 1e12 if cache_ms > 0 else None
    # Query kernel bytes per query: record 64 + slot 4 + throughput 16 + radiance 32 (read
    # and write) + 16 levels x 8 corners x 4 B of hash features.
    qbytes = 64 + 4 + 16 + 32 + 16 * 8 * 4
    out = {"workload": f"learned radiance cache: large scene {cam.width}x{cam.height}, 16 spp, depth 8, one training round per "
                       "frame (2^16 records, 4 Adam steps) then the cached render (queries at vertex 2); hash grid 16 levels x "
                       "2^19 x 2 FP16, 5x64 BF16 MLP, FP32 accumulation",
           "value": paths / (sum(cached_ms) / 1000.0), "unit": "paths/s", "steps": steps, "warmup": warmup,
           "plain": {"value": paths / (sum(plain_ms) / 1000.0), "unit": "paths/s", "ms_per_frame": sum(plain_ms) / steps},
           "speedup_vs_plain": sum(plain_ms) / sum(cached_ms),
           "per_frame_ms": {"train": sum(train_ms) / steps, "train_parts": train_parts,
                            "cached_render": (sum(cached_ms) - sum(train_ms)) / steps,
                            "plain_render": sum(plain_ms) / steps, "tlas_build": sum(build_ms) / steps},
           "extension_rays_per_path": {"cached": rays_cached / paths, "plain": rays_plain / paths},
           "roofline": {"bound": "tensor", "kernel": "k_nrc_forward<query> (fused hash encoding + 5-layer MLP)",
                        "achieved": tflops, "peak": pk["bf16_tflops"], "peak_source": pk["source"], "unit": "TFLOP/s",
                        "frac": (tflops / pk["bf16_tflops"]) if tflops else None, "traffic": None,
                        "queries": queries, "kernel_ms": cache_ms,
                        "hbm_view": {"bytes_per_query": qbytes,
                                     "achieved_gbs": qbytes * queries / (cache_ms / 1000.0) / 1e9 if cache_ms else None,
                                     "peak_gbs": pk["hbm_gbs"]}},
           "clocks": clocks.summary()}
    if errors:
        h16 = cam.height // 16 * 16
        ref = s.render(Profile.reference_transport(depth, ref_spp, seed=7)).image[..., :3]
        conv = k.render(Profile.reference_transport(depth, 256, seed=3)).image[..., :3]
        out["error_vs_plain_ref"] = {"ref_spp": ref_spp, "cached_16spp": _errors(last_cached, ref, h16),
                                     "plain_16spp": _errors(last_plain, ref, h16), "cached_256spp": _errors(conv, ref, h16)}
        # Time to image at equal error: the fewest samples per pixel whose 16x16-block
        # relative RMSE against the reference is <= 1%, and the device time it takes (the
        # cached side adds this frame's training round).
        tti = {}
        for name, fn in (("plain", lambda spp: s.render(Profile.reference_transport(depth, spp, seed=5))),
                         ("cached", lambda spp: k.render(Profile.reference_transport(depth, spp, seed=5)))):
            row = None
            for spp in (8, 12, 16, 24, 32, 48, 64, 96, 128):
                res = fn(spp)
                e = _errors(res.image[..., :3], ref, h16)
                if e["rel_rmse_16x16_blocks"] <= 0.01:
                    ms = res.stats["render_ms"] + (out["per_frame_ms"]["train"] if name == "cached" else 0.0)
                    row = {"spp": spp, "ms": ms, **e}
                    break
            tti[name] = row
        if tti["plain"] and tti["cached"]:
            tti["speedup"] = tti["plain"]["ms"] / tti["cached"]["ms"]
        out["time_to_1pct_block_rmse"] = tti
        # FP64 oracle on the 64x64 centre crop of the last frame (plain path tracing, 64 spp).
        try:
            import dataclasses
            from oracle import pyoracle
            osc = dataclasses.replace(sc, instance_rows=frames[(warmup + steps - 1) % len(frames)].reshape(-1, 3, 4))
            o = pyoracle.OracleScene(osc, fp32=False, fp64=True)
            x0, y0 = cam.width // 2 - 32, cam.height // 2 - 32
            t0 = time.perf_counter()
            oimg, _ = o.render(Profile.reference_transport(depth, 64, seed=11).c(), x0, y0, 64, 64, fp64=True,
                               threads=os.cpu_count() or 1)
            dt = time.perf_counter() - t0
            o.close()
            om = float(oimg[..., :3].mean())
            crop = lambda im: float(im[y0:y0 + 64, x0:x0 + 64].mean())
            out["error_vs_fp64_oracle_crop"] = {"spp": 64, "seconds": dt, "oracle_mean": om,
                                                "cached_256spp_rel_err": crop(conv) / om - 1.0,
                                                f"plain_{ref_spp}spp_rel_err": crop(ref) / om - 1.0}
        except Exception as e:  # reported, never silently dropped
            out["error_vs_fp64_oracle_crop"] = {"error": repr(e)}
    k.close()
    out["block_wall_s"] = time.perf_counter() - t_block
    return out


def _line(value, unit, steps, warmup, ms_per_step, cfg, dtype="f32", **extra):
    return {"metric": METRIC, "value": value, "unit": unit, "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": "synthetic (seeded generator; no dataset)", "config": cfg, **extra}


def run_batch(args, device):
    from vork_b200 import Renderer
    from vork_b200.build import build
    build()
    with Renderer(device) as r:
        blk = batch_block(r, args.jobs, args.warmup)
    print(json.dumps(_line(blk["value"], "paths/s", 1, args.warmup, blk["makespan_ms"],
                           {"workload": blk["workload"], "global_batch": blk["paths"]}, batch=blk,
                           gpu_launches=blk["gpu_launches"], clocks=blk["clocks"])), flush=True)


def run_serve(args, device):
    from vork_b200 import Renderer, scene
    from vork_b200.build import build
    build()
    rates = [float(x) for x in args.rates.split(",")]
    with Renderer(device) as r:
        sc, flock = scene.flock_scene()
        inst = r.install(sc)
        blk = serve_block(r, args.requests, rates, args.schedule, fifo=True, flock_inst=inst, flock=flock,
                          wave_slots=args.serve_wave_slots, serial=args.serve_serial)
        inst.close()
    best = max(blk["rates"], key=lambda x: x["continuous"]["throughput_paths_s"])
    print(json.dumps(_line(best["continuous"]["throughput_paths_s"], "paths/s", len(rates), 0,
                           1000 * best["continuous"]["wall_s"], {"workload": blk["workload"]}, serve=blk)), flush=True)


def run_cache(args, device):
    from vork_b200 import Renderer, scene
    from vork_b200.build import build
    build()
    w, h = (int(v) for v in args.res.lower().split("x"))
    sc, flock = scene.flock_scene(seed=0, width=w, height=h)
    frames = frames_for(sc, flock, args.warmup + args.steps)
    with Renderer(device) as r:
        s = r.install(sc)
        blk = cache_block(r, s, sc, frames, args.warmup, args.steps, errors=not args.no_error)
        s.close()
    print(json.dumps(_line(blk["value"], "paths/s", args.steps, args.warmup, 1000 * 16 * w * h / blk["value"],
                           {"workload": blk["workload"], "global_batch": w * h * 16,
                            "l2_flush": "inputs > L2: 1M-instance TLAS + 2M-tri BLAS + wavefront queues per frame"},
                           dtype="f32+bf16", cache=blk, roofline=blk["roofline"], clocks=blk["clocks"])), flush=True)


def max_over_ranks(value: float, dist, device=None) -> float:
    """The largest of every rank's value (NCCL needs a CUDA tensor, gloo a host one)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_dry(args, rank, world):
    """The multi-rank host logic of the replicas bench without a GPU (gloo): rendezvous,
    a different seeded workload per rank, barrier, a stand-in step time per rank, the
    max over ranks and one JSON line from rank 0."""
    import datetime
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        dist.barrier()
    sc, _, prof, cfg = workload("small", seed=rank)
    paths_per_step = sc.camera.width * sc.camera.height * prof.samples
    elapsed_ms = args.steps * 10.0 * (1 + rank)          # stand-in device time of this rank
    elapsed = max_over_ranks(elapsed_ms, dist)
    digest = float(np.asarray(sc.instance_rows, np.float64).sum())
    digests = [digest]
    if dist is not None:
        out = [None] * world
        dist.all_gather_object(out, digest)
        digests = out
    if rank == 0:
        print(json.dumps({"dry_run": True, "n_gpus": world, "steps": args.steps, "ms_per_step": elapsed / args.steps,
                          "value": world * args.steps * paths_per_step / (elapsed / 1000.0), "unit": "paths/s",
                          "scaling": "weak", "rank_workload_digests": digests, "config": cfg}), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vkb", choices=["vkb", "reference"])
    ap.add_argument("--config", default="large", choices=["large", "small", "profile", "batch", "serve", "cache"])
    ap.add_argument("--jobs", type=int, default=256, help="batch: preview jobs")
    ap.add_argument("--requests", type=int, default=200, help="serve: requests per arrival rate")
    ap.add_argument("--rates", default="1,5,20,50", help="serve: Poisson arrival rates (req/s)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tlas", choices=["lbvh", "ploc"], default="lbvh", help="TLAS builder of the frame scene")
    ap.add_argument("--blas", choices=["4", "8"], default="4", help="BLAS nodes: 4-wide FP32 planes or compressed 8-wide")
    ap.add_argument("--blas-builder", choices=["sah", "lbvh", "ploc"], default="sah", help="BLAS build: host SAH or GPU LBVH / PLOC")
    ap.add_argument("--serial-waves", action="store_true", help="large: one wave after another on one stream (no overlap)")
    ap.add_argument("--wave-samples", type=int, default=0, help="large: samples per wave (0: as many as the wavefront holds)")
    ap.add_argument("--serve-wave-slots", type=int, default=0, help="serve: path slots per server wave (0: the context's)")
    ap.add_argument("--serve-serial", action="store_true", help="serve: the server's waves on one stream (replayed graphs)")
    ap.add_argument("--no-error", action="store_true", help="cache: skip the reference renders (timing/profiling runs)")
    ap.add_argument("--res", default="1920x1080", help="cache: frame resolution (smaller for profiling captures)")
    ap.add_argument("--schedule", default="srpt", choices=["srpt", "aged", "fair", "packed"], help="serve: wave schedule")
    ap.add_argument("--dry-run", action="store_true", help="multi-rank host logic on CPU (gloo), no GPU work")
    ap.add_argument("--no-blocks", action="store_true", help="large: skip the batch/cache/serve blocks after the frame timing")
    ap.add_argument("--block-requests", type=int, default=40, help="large: requests of the serve block")
    ap.add_argument("--block-rate", type=float, default=2.0, help="large: arrival rate of the serve block (req/s)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.dry_run:
        return run_dry(args, rank, world)
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.config == "batch":
        return run_batch(args, local)
    if args.config == "serve":
        return run_serve(args, local)
    if args.config == "cache":
        return run_cache(args, local)

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)

    from vork_b200 import Renderer, abi
    from vork_b200.build import build
    if rank == 0:
        build()
    if dist:
        dist.barrier()

    sc, flock, prof, cfg = workload(args.config, seed=rank)
    sc.tlas_builder = abi.TLAS_PLOC if args.tlas == "ploc" else abi.TLAS_LBVH
    sc.blas_format = abi.BLAS_WIDE8 if args.blas == "8" else abi.BLAS_WIDE4
    sc.blas_builder = {"sah": abi.BLAS_BUILD_SAH, "lbvh": abi.BLAS_BUILD_LBVH, "ploc": abi.BLAS_BUILD_PLOC}[args.blas_builder]
    frames = frames_for(sc, flock, args.warmup + args.steps)
    cam = sc.camera
    npix = cam.width * cam.height
    paths_per_step = npix * prof.samples
    r = Renderer(local)
    s = r.install(sc)
    info0 = s.info()
    install = {k: info0[k] for k in ("install_ms", "blas_host_ms", "upload_ms", "tlas_ms", "scene_bytes", "num_triangles",
                                     "num_instances")}
    stream = torch.cuda.ExternalStream(r.stream, device=torch.device("cuda", local))
    dev_frames = [torch.from_numpy(f).to(f"cuda:{local}") for f in frames]
    pinned = [torch.from_numpy(f).pin_memory() for f in frames]
    image = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device=f"cuda:{local}")
    host_image = torch.empty((cam.height, cam.width, 4), dtype=torch.float32).pin_memory()
    serial = abi.PROFILE_SERIAL_WAVES if args.serial_waves else 0
    prof = prof.__class__(**{**prof.__dict__, "flags": serial, "wave_samples": args.wave_samples})
    # Kernel durations for the roofline come from one more frame with events around every
    # closest-hit launch and its waves one after another: with overlapped waves an event
    # pair would also count the other stream's kernels sharing the SMs.
    kernel_prof = prof.__class__(**{**prof.__dict__, "flags": abi.PROFILE_TIME_KERNELS | abi.PROFILE_SERIAL_WAVES})
    n_inst = frames[0].shape[0]

    def step(i, p):
        s.update_instances_device(dev_frames[i].data_ptr(), n_inst, 1)
        return s.render(p, device_ptr=image.data_ptr())

    def sync():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    for i in range(args.warmup):
        step(i, prof)
    # One instrumented render (untimed) for the roofline's algorithmic bytes.
    counted = s.render(prof.__class__(**{**prof.__dict__, "flags": abi.PROFILE_COUNT_TRAVERSAL | serial}), device_ptr=image.data_ptr()).stats

    sync()
    launches0 = s.launch_count
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    trace_ms = 0.0
    trace_launches = 0
    build_ms = 0.0
    latencies = []
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for k in range(args.steps):
            st = step(args.warmup + k, prof).stats
            latencies.append(st["render_ms"] + st["build_ms"])
            build_ms += st["build_ms"]
        ev1.record(stream)
        sync()
    elapsed_ms = ev0.elapsed_time(ev1)
    launches = s.launch_count - launches0
    # The kernel-timing frame (untimed; the last frame's rows again).
    kt = step(args.warmup + args.steps - 1, kernel_prof).stats
    trace_ms, trace_launches = kt["trace_ms"] * args.steps, kt["trace_launches"] * args.steps
    tlas = {"builder": ("PLOC (radius 16)" if args.tlas == "ploc" else "Karras LBVH") + " over 30-bit Morton order (bit 30: boxes wider than a quarter of the centroid spread, split at the root), rebuilt every frame",
            "build_ms_per_frame": build_ms / args.steps,
            "blas_nodes": "compressed 8-wide (80 B)" if args.blas == "8" else "4-wide FP32 planes (128 B)",
            "blas_builder": {"sah": "binned SAH on the host threads", "lbvh": "GPU LBVH", "ploc": "GPU PLOC"}[args.blas_builder],
            **s.tlas_stats()}
    elapsed_ms = max_over_ranks(elapsed_ms, dist, f"cuda:{local}")
    value = world * args.steps * paths_per_step / (elapsed_ms / 1000.0)

    # e2e: pinned host rows in, host image out, through the C ABI (copies inside the call).
    sync()
    t0 = time.perf_counter()
    for k in range(args.steps):
        s.update_instances(pinned[args.warmup + k].numpy(), policy=1)
        s.render(prof, out=host_image.numpy())
    sync()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist, f"cuda:{local}")
    e2e = world * args.steps * paths_per_step / e2e_s

    if rank == 0:
        pk = peaks()
        alg_bytes = roofline_bytes(counted)
        trace_s_per_frame = trace_ms / args.steps / 1000.0
        achieved_gbs = alg_bytes / trace_s_per_frame / 1e9 if trace_ms > 0 else None
        stored_gbs = stored_bytes(counted) / trace_s_per_frame / 1e9 if trace_ms > 0 else None
        launches_per_frame = trace_launches / args.steps
        traffic = dram_gbs = None
        prof_note = ROOT / "profiles" / "trace_closest_traffic.json"
        if prof_note.exists() and args.config in ("large", "profile"):
            # ncu capture of every closest-hit launch of one timed frame of this workload
            # (DRAM bytes per ray, times this run's rays per launch).
            tr = json.loads(prof_note.read_text())
            rays_per_launch = counted["extension_rays"] / max(1, counted["trace_launches"])
            traffic = tr["traffic_bytes_per_ray"] * rays_per_launch
            if trace_ms > 0:
                dram_gbs = traffic * launches_per_frame / trace_s_per_frame / 1e9
        limiter = trace_limiter()
        line = {
            "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded generator; no dataset)",
            "config": {**cfg, "global_batch": paths_per_step * world, "parallelism": f"replicas x{world}",
                       "waves": "one stream" if args.serial_waves else "alternating between two streams (overlapped)",
                       "l2_flush": "inputs > L2: 1M-instance TLAS + 2M-tri BLAS + 1.1 GB of wavefront queues per frame"},
            "latency_ms": {"p50": float(np.percentile(latencies, 50)), "p99": float(np.percentile(latencies, 99))},
            # Against HBM (the only roofline family this integer/pointer-chasing kernel has);
            # `frac` counts algorithmic bytes (80 B per node visit, 36 B per triangle, 64 B per
            # instance entry, 56 B per ray).  The hardware serves most node fetches from L1/L2,
            # so `dram_frac` (measured DRAM bytes) is far lower and `limiter` names what ncu
            # shows actually bounds the kernel.
            "roofline": {"bound": "hbm", "kernel": "k_trace<closest>", "achieved": achieved_gbs, "peak": pk["hbm_gbs"],
                         "peak_source": pk["source"], "unit": "GB/s",
                         "frac": (achieved_gbs / pk["hbm_gbs"]) if achieved_gbs else None, "traffic": traffic,
                         "bytes_per_unit": {"node_visit": NODE_BYTES, "triangle_test": TRI_BYTES, "instance_entry": INSTANCE_BYTES,
                                            "ray": RAY_BYTES},
                         "frac_at_stored_node_bytes": (stored_gbs / pk["hbm_gbs"]) if stored_gbs else None,
                         "dram_gbs": dram_gbs, "dram_frac": (dram_gbs / pk["hbm_gbs"]) if dram_gbs else None,
                         "limiter": limiter,
                         "algorithmic_bytes_per_launch": alg_bytes / max(1.0, launches_per_frame),
                         "algorithmic_bytes_per_frame": alg_bytes, "trace_ms_per_frame": trace_ms / args.steps,
                         "trace_launches_per_frame": trace_launches / args.steps,
                         "share_of_step": trace_ms / elapsed_ms if elapsed_ms else None},
            "e2e": {"value": e2e, "unit": "paths/s", "h2d_bytes_per_step": int(frames[0].nbytes),
                    "d2h_bytes_per_step": int(npix * 16)},
            "gpu_launches": int(launches),
            "tlas": tlas,
            "install": install,
            "clocks": clocks.summary(),
            "work": {k: counted[k] for k in ("extension_rays", "shadow_rays", "nodes_visited", "triangles_tested",
                                             "instances_entered", "blas_nodes_visited", "shadow_nodes_visited", "shadow_triangles_tested",
                                             "traversal_overflows", "dropped_path_samples")},
        }
        if not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline(args.config)
            except Exception as e:  # reported, never silently dropped
                line["cpu_baseline"] = {"value": None, "error": repr(e)}
        if world == 1 and args.config == "large" and not args.no_blocks:
            # The other configurations, compact, each with its own clock record: batched
            # previews (256 jobs), the learned cache on this frame scene, and serving at one
            # arrival rate with the plain FIFO baseline on the same trace.
            for name, fn in (("small", lambda: small_block(r)),
                             ("batch", lambda: batch_block(r, 256, 1)),
                             ("cache", lambda: cache_block(r, s, sc, frames, 2, 3)),
                             ("serve", lambda: serve_block(r, args.block_requests, [args.block_rate], fifo=True,
                                                           flock_inst=s, flock=flock))):
                try:
                    line[name] = fn()
                except Exception as e:  # reported, never silently dropped
                    line[name] = {"error": repr(e)}
        print(json.dumps(line), flush=True)
    s.close()
    r.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
