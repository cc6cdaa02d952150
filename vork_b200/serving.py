"""Serving front end over vkb_server_*: continuous batching with memory admission.

`Server` wraps the C ABI; `poisson_load` drives it with seeded Poisson arrivals and
reports p50/p99 latency and throughput.  Requests reference installed (resident)
scenes; a sequence request is `frames` consecutive renders of its scene with
per-frame seeds.
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
    def __init__(self, renderer, memory_budget_bytes: int = 160 << 30, max_jobs: int = 64, flags: int = 0, wave_capacity: int = 0):
        self.r = renderer
        cfg = abi.VkbServerConfig()
        cfg.memory_budget_bytes, cfg.max_jobs, cfg.flags, cfg.wave_capacity = memory_budget_bytes, max_jobs, flags, wave_capacity
        h = C.c_void_p()
        abi.check(renderer.lib.vkb_server_create(renderer.h, C.byref(cfg), C.byref(h)))
        self.h = h
        self.images: dict[int, np.ndarray] = {}

    def submit(self, installed, profile: Profile) -> int:
        cam = installed.scene.camera
        img = np.empty((cam.height, cam.width, 4), np.float32)
        rid = C.c_uint64()
        p = profile.c()
        abi.check(self.r.lib.vkb_server_submit(self.h, installed.h, C.byref(p), abi.fptr(img), C.byref(rid)))
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
    ids: list = field(default_factory=list)
    done_at: float | None = None


def request_mix(count: int, scene_count: int, seed: int = 0, still_fraction: float = 0.8, frames: int = 24,
                spp_range=(8, 128), bounces: int = 8):
    """Seeded request mix: 80% stills / 20% sequences of `frames` frames, spp U{lo..hi},
    scene chosen uniformly among the installed resident scenes."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        spp = int(rng.integers(spp_range[0], spp_range[1] + 1))
        prof = Profile.reference_transport(bounces, spp, seed=int(rng.integers(0, 1 << 31)))
        nframes = 1 if rng.random() < still_fraction else frames
        out.append(Request(int(rng.integers(0, scene_count)), prof, nframes, 0.0))
    return out


def poisson_load(server: Server, scenes: list, requests: list, rate: float, seed: int = 0, timeout_s: float = 600.0) -> dict:
    """Submit `requests` with Poisson arrivals at `rate` per second (wall clock), stepping
    the server between arrivals; latency = completion - arrival of each request."""
    rng = np.random.default_rng(seed)
    t = 0.0
    for r in requests:
        t += rng.exponential(1.0 / rate)
        r.arrival = t
    start = time.perf_counter()
    pending = list(requests)
    running: list[Request] = []
    paths = 0
    while pending or running:
        now = time.perf_counter() - start
        if now > timeout_s:
            raise RuntimeError("serving run exceeded its time limit")
        while pending and pending[0].arrival <= now:
            r = pending.pop(0)
            inst = scenes[r.scene_index]
            for f in range(r.frames):
                prof = Profile(**{**r.profile.__dict__, "seed": (r.profile.seed + 7919 * f) & 0x7FFFFFFF})
                r.ids.append(server.submit(inst, prof))
                paths += inst.scene.camera.width * inst.scene.camera.height * prof.samples
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
                r.done_at = now
            else:
                still.append(r)
        running = still
    wall = time.perf_counter() - start
    lat = np.array([r.done_at - r.arrival for r in requests])
    return {"requests": len(requests), "rate": rate, "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "throughput_paths_s": paths / wall, "wall_s": wall}
