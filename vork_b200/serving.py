"""Serving front end over vkb_server_*: continuous batching with memory admission.

`Server` wraps the C ABI; `poisson_load` drives it with seeded Poisson arrivals and
reports p50/p99 latency and throughput; `fifo_load` serves the same arrivals with the
plain path one request at a time, the baseline.  Requests reference installed
(resident) scenes, each at its own resolution; a sequence request is `frames`
consecutive renders with per-frame seeds, and on an animated scene each frame renders
through a fork of the scene whose TLAS is rebuilt from that frame's instance rows.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi
from . import Profile


class Server:
    def __init__(self, renderer, memory_budget_bytes: int = 160 << 30, max_jobs: int = 64, flags: int = 0, wave_capacity: int = 0,
                 aging_paths_per_s: float = 0.0):
        self.r = renderer
        cfg = abi.VkbServerConfig()
        cfg.memory_budget_bytes, cfg.max_jobs, cfg.flags, cfg.wave_capacity = memory_budget_bytes, max_jobs, flags, wave_capacity
        cfg.aging_paths_per_s = aging_paths_per_s
        h = C.c_void_p()
        abi.check(renderer.lib.vkb_server_create(renderer.h, C.byref(cfg), C.byref(h)))
        self.h = h
        self.images: dict[int, np.ndarray] = {}

    def submit(self, installed, profile: Profile, camera: abi.VkbCamera | None = None) -> int:
        """Queue a request (vkb_server_submit_view): the scene through `camera` (its
        resolution sets the image's), or through the scene's own camera."""
        cam = camera if camera is not None else installed.scene.camera
        img = np.empty((cam.height, cam.width, 4), np.float32)
        rid = C.c_uint64()
        p = profile.c()
        cptr = C.cast(C.byref(camera), C.c_void_p) if camera is not None else None
        abi.check(self.r.lib.vkb_server_submit_view(self.h, installed.h, cptr, C.byref(p), abi.fptr(img), C.byref(rid)))
        self.images[rid.value] = img
        return rid.value

    def step(self) -> dict:
        st = abi.VkbServerStatus()
        abi.check(self.r.lib.vkb_server_step(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in abi.VkbServerStatus._fields_ if k != "reserved"}

    def state(self, rid: int) -> int:
        s = C.c_int()
        abi.check(self.r.lib.vkb_server_poll(self.h, rid, C.byref(s)))
        return s.value

    def run_until_idle(self, max_steps: int = 1_000_000):
        for _ in range(max_steps):
            st = self.step()
            if st["queued"] == 0 and st["running"] == 0:
                return
        raise RuntimeError("server did not drain")

    def close(self):
        if self.h:
            self.r.lib.vkb_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


@dataclass
class Request:
    scene_index: int
    profile: Profile
    frames: int
    arrival: float
    width: int = 0                  # 0: the scene camera's resolution
    height: int = 0
    ids: list = field(default_factory=list)
    done_at: float | None = None
    next_frame: int = 0
    fork: object = None


def request_mix(count: int, scene_count: int, seed: int = 0, still_fraction: float = 0.8, frames: int = 24,
                spp_range=(8, 128), bounces: int = 8, pixels_range=None):
    """Seeded request mix: 80% stills / 20% sequences of `frames` frames, spp U{lo..hi},
    scene chosen uniformly among the installed resident scenes; with `pixels_range`
    (lo, hi), a resolution per request whose pixel count is log-uniform in it, at an
    aspect of 1, 4/3 or 16/9 (at most 1920x1080)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        spp = int(rng.integers(spp_range[0], spp_range[1] + 1))
        prof = Profile.reference_transport(bounces, spp, seed=int(rng.integers(0, 1 << 31)))
        nframes = 1 if rng.random() < still_fraction else frames
        req = Request(int(rng.integers(0, scene_count)), prof, nframes, 0.0)
        if pixels_range is not None:
            px = math.exp(rng.uniform(math.log(pixels_range[0]), math.log(pixels_range[1])))
            aspect = float(rng.choice([1.0, 4.0 / 3.0, 16.0 / 9.0]))
            req.width = int(min(1920, max(16, round(math.sqrt(px * aspect)))))
            req.height = int(min(1080, max(16, round(math.sqrt(px / aspect)))))
        out.append(req)
    return out


def view(camera: abi.VkbCamera, width: int, height: int) -> abi.VkbCamera:
    """The same pinhole at another resolution (vertical field of view kept)."""
    c = abi.VkbCamera()
    C.pointer(c)[0] = camera
    c.width, c.height = width, height
    c.proj_x = camera.proj_y / (width / height)
    return c


def _frame_profile(r: Request, f: int) -> Profile:
    return Profile(**{**r.profile.__dict__, "seed": (r.profile.seed + 7919 * f) & 0x7FFFFFFF})


def _camera(r: Request, inst):
    return view(inst.scene.camera, r.width, r.height) if r.width else None


def _paths(r: Request, inst) -> int:
    cam = inst.scene.camera
    w, h = (r.width, r.height) if r.width else (cam.width, cam.height)
    return w * h * r.profile.samples * r.frames


def _arrivals(requests, rate, seed):
    rng = np.random.default_rng(seed)
    t = 0.0
    for r in requests:
        t += rng.exponential(1.0 / rate)
        r.arrival = t
        r.ids, r.done_at, r.next_frame, r.fork = [], None, 0, None


def _summary(requests, rate, paths, wall):
    lat = np.array([r.done_at - r.arrival for r in requests])
    return {"requests": len(requests), "rate": rate, "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "throughput_paths_s": paths / wall, "wall_s": wall}


def poisson_load(server: Server, scenes: list, requests: list, rate: float, seed: int = 0, timeout_s: float = 600.0,
                 animations: dict | None = None) -> dict:
    """Submit `requests` with Poisson arrivals at `rate` per second (wall clock), stepping
    the server between arrivals (continuous batching); latency = completion - arrival.

    `animations` maps a scene index to its per-frame instance rows: a sequence on such a
    scene renders through its own fork of the scene, whose TLAS is rebuilt from frame
    f's rows before frame f is submitted (frames in order, each after the previous one
    finished, while other requests keep sharing the waves)."""
    animations = animations or {}
    _arrivals(requests, rate, seed)
    start = time.perf_counter()
    pending = list(requests)
    running: list[Request] = []
    paths = 0

    def submit_frame(r: Request):
        inst = r.fork if r.fork is not None else scenes[r.scene_index]
        f = r.next_frame
        if r.fork is not None:
            rows = animations[r.scene_index]
            r.fork.update_instances(rows[f % len(rows)], policy=1)
        r.ids.append(server.submit(inst, _frame_profile(r, f), _camera(r, inst)))
        r.next_frame += 1

    try:
        while pending or running:
            now = time.perf_counter() - start
            if now > timeout_s:
                raise RuntimeError("serving run exceeded its time limit")
            while pending and pending[0].arrival <= now:
                r = pending.pop(0)
                inst = scenes[r.scene_index]
                paths += _paths(r, inst)
                if r.frames > 1 and r.scene_index in animations:
                    r.fork = inst.fork()
                    submit_frame(r)                 # frame by frame through the fork
                else:
                    while r.next_frame < r.frames:
                        submit_frame(r)
                running.append(r)
            if not running:
                if pending:
                    time.sleep(max(0.0, min(pending[0].arrival - now, 0.05)))
                continue
            server.step()
            now = time.perf_counter() - start
            still = []
            for r in running:
                if all(server.state(i) == 2 for i in r.ids):
                    if r.next_frame < r.frames:
                        submit_frame(r)
                        still.append(r)
                        continue
                    r.done_at = now
                    if r.fork is not None:
                        r.fork.close()
                        r.fork = None
                else:
                    still.append(r)
            running = still
    finally:
        for r in requests:
            if r.fork is not None:
                server.run_until_idle()
                r.fork.close()
                r.fork = None
    return _summary(requests, rate, paths, time.perf_counter() - start)


def fifo_load(scenes: list, requests: list, rate: float, seed: int = 0, timeout_s: float = 600.0,
              animations: dict | None = None) -> dict:
    """The plain path served one request at a time in arrival order (vork's kept-alive
    session, crates/vork-cli/src/session.rs:1-60): the same arrival trace and work as
    `poisson_load`, each frame a plain vkb_render_view call; latency = completion - arrival."""
    animations = animations or {}
    _arrivals(requests, rate, seed)
    start = time.perf_counter()
    paths = 0
    for r in requests:
        now = time.perf_counter() - start
        if now > timeout_s:
            raise RuntimeError("serving run exceeded its time limit")
        if r.arrival > now:
            time.sleep(r.arrival - now)
        inst = scenes[r.scene_index]
        paths += _paths(r, inst)
        fork = inst.fork() if (r.frames > 1 and r.scene_index in animations) else None
        try:
            target = fork if fork is not None else inst
            cam = _camera(r, inst)
            for f in range(r.frames):
                if fork is not None:
                    rows = animations[r.scene_index]
                    fork.update_instances(rows[f % len(rows)], policy=1)
                target.render(_frame_profile(r, f), camera=cam)
        finally:
            if fork is not None:
                fork.close()
        r.done_at = time.perf_counter() - start
    return _summary(requests, rate, paths, time.perf_counter() - start)
