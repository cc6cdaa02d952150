"""vork_b200: a B200 (sm_100a) render backend for vork's `std/path` integrator.

The product path is the CUDA library behind include/vkb.h; this module is the
host-side mirror of the reference's entry (`Shot::render` / `vork.render(scene, ...)`,
crates/vork-render/src/shot.rs:374, packages/python/vork/__init__.py:291) over it.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .abi import VkbError
from .scene import Scene

__all__ = ["Profile", "Renderer", "InstalledScene", "RadianceCache", "render", "VkbError", "Scene"]


@dataclass
class Profile:
    """PathSettings of one render (passes/path.rs:576-607; constants.rs:256-267).

    The defaults are vork's std/path defaults; `reference_transport(depth)` is the
    reference's own test hook `reference_transport_bounces` (passes/path.rs:599-607):
    every bounce budget = depth, transparent = depth, both clamps off.
    """
    samples: int = 64
    seed: int = 0
    bounces: tuple = (12, 4, 4, 12)
    transparent: int = 8
    caustics: int = 0b11
    clamp_direct: float = 0.0
    clamp_indirect: float = 10.0
    light_threshold: float = 0.01
    adaptive: bool = False
    adaptive_threshold: float = 0.0
    adaptive_min_samples: int = 0
    first_sample: int = 0
    sample_count: int = 0
    wave_samples: int = 0
    flags: int = 0

    @classmethod
    def reference_transport(cls, depth: int, samples: int, seed: int = 0, **kw) -> "Profile":
        return cls(samples=samples, seed=seed, bounces=(depth,) * 4, transparent=depth, clamp_direct=0.0,
                   clamp_indirect=0.0, **kw)

    def c(self) -> abi.VkbProfile:
        p = abi.VkbProfile()
        p.samples, p.first_sample, p.sample_count, p.seed = self.samples, self.first_sample, self.sample_count, self.seed & 0xFFFFFFFF
        p.bounces[:] = list(self.bounces)
        p.transparent, p.caustics = self.transparent, self.caustics
        p.clamp_direct, p.clamp_indirect, p.light_threshold = self.clamp_direct, self.clamp_indirect, self.light_threshold
        p.adaptive = 1 if self.adaptive else 0
        p.adaptive_threshold, p.adaptive_min_samples = self.adaptive_threshold, self.adaptive_min_samples
        p.wave_samples = self.wave_samples
        p.flags = self.flags
        return p


class Renderer:
    """One CUDA device (Renderer::new, crates/vork-render/src/lib.rs:726)."""

    def __init__(self, device: int = 0):
        self.lib = abi.load()
        h = C.c_void_p()
        abi.check(self.lib.vkb_open(device, C.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            self.lib.vkb_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def install(self, scene: Scene) -> "InstalledScene":
        return InstalledScene(self, scene)

    def sampler_groups(self, px, py, index, groups, count, stream):
        px, py, index, groups = (np.ascontiguousarray(a, np.uint32) for a in (px, py, index, groups))
        out = np.zeros((px.size, 4), np.uint32)
        abi.check(self.lib.vkb_debug_sampler_groups(self.h, px.size, abi.uptr(px), abi.uptr(py), abi.uptr(index), abi.uptr(groups),
                                                    count, stream, abi.uptr(out)))
        return out

    def render_batch(self, items, flags: int = 0, outs=None):
        """Render [(InstalledScene, Profile), ...] together (vkb_render_batch): one shared
        wavefront, per-job images identical to InstalledScene.render.  `outs`, when given,
        are the (H, W, 4) float32 host images to fill (else new ones are made)."""
        n = len(items)
        jobs = (abi.VkbJob * max(1, n))()
        images = []
        for k, (inst, prof) in enumerate(items):
            cam = inst.scene.camera
            img = outs[k] if outs is not None else np.empty((cam.height, cam.width, 4), np.float32)
            assert img.shape == (cam.height, cam.width, 4) and img.dtype == np.float32 and img.flags.c_contiguous
            images.append(img)
            jobs[k].scene = inst.h
            jobs[k].profile = prof.c()
            jobs[k].out.rgba = img.ctypes.data_as(C.c_void_p)
            jobs[k].out.on_device = 0
        st = abi.VkbStats()
        abi.check(self.lib.vkb_render_batch(self.h, jobs, n, flags, C.byref(st)))
        return images, {k: getattr(st, k) for k, _ in abi.VkbStats._fields_}

    def autotune(self, items) -> dict:
        """Pick the wave capacity and trace grid for these jobs (vkb_autotune)."""
        n = len(items)
        jobs = (abi.VkbJob * max(1, n))()
        for k, (inst, prof) in enumerate(items):
            jobs[k].scene = inst.h
            jobs[k].profile = prof.c()
        r = abi.VkbTuneResult()
        abi.check(self.lib.vkb_autotune(self.h, jobs, n, C.byref(r)))
        return {"best_capacity": r.best_capacity, "best_blocks_per_sm": r.best_blocks_per_sm, "best_ms": r.best_ms,
                "tried": [(r.capacity[i], r.blocks_per_sm[i], r.ms[i]) for i in range(min(r.tried, 16))]}

    @property
    def stream(self) -> int:
        """The cudaStream_t (as an integer) this device's kernels run on."""
        return int(self.lib.vkb_ctx_stream(self.h) or 0)

    def brdf_lut(self):
        out = np.zeros((2240, 128, 4), np.float32)
        abi.check(self.lib.vkb_debug_brdf_lut(self.h, abi.fptr(out)))
        return out


@dataclass
class RenderResult:
    image: np.ndarray          # (H, W, 4) linear RGBA32F mean
    stats: dict
    primary_ids: np.ndarray | None = None
    guide_albedo: np.ndarray | None = None   # (H, W, 4): mean guide albedo (rgb) and coverage (w)
    guide_normal: np.ndarray | None = None   # (H, W, 4): mean shading normal (xyz), 0


class InstalledScene:
    """Renderer::install + FrameRays (lib.rs:1322-1470; rt.rs:1098-1385) for one scene."""

    def __init__(self, renderer: Renderer, scene: Scene, _handle=None):
        self.r = renderer
        self.scene = scene
        if _handle is not None:       # a fork: the base's descriptor describes it
            self.desc = None
            self.h = _handle
            return
        self.desc = scene.desc()
        h = C.c_void_p()
        abi.check(renderer.lib.vkb_scene_create(renderer.h, C.byref(self.desc), C.byref(h)))
        self.h = h

    def fork(self) -> "InstalledScene":
        """A frame slot (vkb_scene_fork): shares this scene's meshes, BLASes, materials and
        lights, owns its instance rows and TLAS (starting from this scene's rows)."""
        h = C.c_void_p()
        abi.check(self.r.lib.vkb_scene_fork(self.h, C.byref(h)))
        return InstalledScene(self.r, self.scene, _handle=h)

    def close(self):
        """Release the scene (a base with live forks is refused: close the forks first)."""
        if self.h:
            abi.check(self.r.lib.vkb_scene_destroy(self.h))
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def update_instances(self, rows: np.ndarray, policy: int = 0):
        rows = np.ascontiguousarray(rows, np.float32).reshape(-1)
        abi.check(self.r.lib.vkb_scene_update_instances(self.h, abi.fptr(rows), rows.size // 12, policy))

    def update_instances_device(self, device_ptr: int, count: int, policy: int = 0):
        abi.check(self.r.lib.vkb_scene_update_instances_device(self.h, C.c_void_p(device_ptr), count, policy))

    def info(self) -> dict:
        i = abi.VkbSceneInfo()
        abi.check(self.r.lib.vkb_scene_info(self.h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in abi.VkbSceneInfo._fields_ if k != "reserved"}

    @property
    def launch_count(self) -> int:
        return int(self.r.lib.vkb_scene_launch_count(self.h))

    def render(self, profile: Profile, ids: bool = False, out: np.ndarray | None = None, device_ptr: int | None = None,
               camera: abi.VkbCamera | None = None, guides: bool = False) -> RenderResult:
        """Render under `profile` (vkb_render), or through `camera` instead of the scene's
        own (vkb_render_view: its resolution sets the image's); `guides` also returns the
        denoiser guide planes (host output only)."""
        cam = camera if camera is not None else self.scene.camera
        o = abi.VkbOutput()
        img = None
        if device_ptr is not None:
            o.rgba = C.c_void_p(device_ptr)
            o.on_device = 1
        else:
            img = out if out is not None else np.empty((cam.height, cam.width, 4), np.float32)
            o.rgba = img.ctypes.data_as(C.c_void_p)
            o.on_device = 0
        idbuf = np.empty((cam.height, cam.width, 2), np.uint32) if ids else None
        o.primary_ids = abi.uptr(idbuf) if ids else None
        ga = gn = None
        if guides:
            if device_ptr is not None:
                raise ValueError("guide planes are returned in host memory: render to a host image")
            ga = np.empty((cam.height, cam.width, 4), np.float32)
            gn = np.empty((cam.height, cam.width, 4), np.float32)
            o.guide_albedo = ga.ctypes.data_as(C.c_void_p)
            o.guide_normal = gn.ctypes.data_as(C.c_void_p)
        st = abi.VkbStats()
        p = profile.c()
        if camera is not None:
            abi.check(self.r.lib.vkb_render_view(self.h, C.cast(C.byref(camera), C.c_void_p), C.byref(p), C.byref(o), C.byref(st)))
        else:
            abi.check(self.r.lib.vkb_render(self.h, C.byref(p), C.byref(o), C.byref(st)))
        stats = {k: getattr(st, k) for k, _ in abi.VkbStats._fields_}
        return RenderResult(img, stats, idbuf, ga, gn)

    def tlas_morton(self):
        out = np.zeros(self.scene.instance_rows.shape[0], np.uint32)
        abi.check(self.r.lib.vkb_debug_tlas_morton(self.h, abi.uptr(out)))
        return out

    def blas_morton(self, mesh: int):
        out = np.zeros(self.scene.meshes[mesh].num_triangles, np.uint32)
        abi.check(self.r.lib.vkb_debug_blas_morton(self.h, mesh, abi.uptr(out)))
        return out

    def tlas_stats(self) -> dict:
        """Walk the TLAS (vkb_debug_tlas_stats): validity, deepest leaf, surface area cost."""
        cost, depth, valid = C.c_double(), C.c_uint32(), C.c_uint32()
        abi.check(self.r.lib.vkb_debug_tlas_stats(self.h, C.byref(cost), C.byref(depth), C.byref(valid)))
        return {"valid": bool(valid.value), "max_depth": int(depth.value), "sah_cost": float(cost.value)}

    def trace(self, rays7: np.ndarray):
        r = np.ascontiguousarray(rays7, np.float32)
        n = r.shape[0]
        t = np.zeros(n, np.float32); ids = np.zeros((n, 2), np.uint32); uv = np.zeros((n, 2), np.float32)
        abi.check(self.r.lib.vkb_debug_trace(self.h, n, abi.fptr(r), abi.fptr(t), abi.uptr(ids), abi.fptr(uv)))
        return t, ids, uv

    def occluded(self, rays7: np.ndarray) -> np.ndarray:
        """Any-hit occlusion of (origin, dir, tmax) rays by the shadow-ray traversal: (n,) bool."""
        r = np.ascontiguousarray(rays7, np.float32)
        out = np.zeros(r.shape[0], np.uint32)
        abi.check(self.r.lib.vkb_debug_occluded(self.h, r.shape[0], abi.fptr(r), abi.uptr(out)))
        return out.astype(bool)


class RadianceCache:
    """A learned radiance cache bound to an installed scene (vkb_cache_*)."""

    def __init__(self, installed: "InstalledScene", **config):
        self.scene = installed
        self.r = installed.r
        cfg = abi.VkbCacheConfig()
        for k, v in config.items():
            setattr(cfg, k, v)
        h = C.c_void_p()
        abi.check(self.r.lib.vkb_cache_create(installed.h, C.byref(cfg), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.r.lib.vkb_cache_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def train(self, profile: Profile) -> dict:
        """One online training round (vkb_cache_train) with the profile's bounce limits and seed."""
        st = abi.VkbCacheStats()
        p = profile.c()
        abi.check(self.r.lib.vkb_cache_train(self.h, C.byref(p), C.byref(st)))
        return {k: getattr(st, k) for k, _ in abi.VkbCacheStats._fields_}

    def render(self, profile: Profile) -> "RenderResult":
        """Render the scene through the cache (vkb_render_cached) into a host image."""
        cam = self.scene.scene.camera
        img = np.empty((cam.height, cam.width, 4), np.float32)
        o = abi.VkbOutput()
        o.rgba = img.ctypes.data_as(C.c_void_p)
        o.on_device = 0
        st = abi.VkbStats()
        p = profile.c()
        abi.check(self.r.lib.vkb_render_cached(self.h, C.byref(p), C.byref(o), C.byref(st)))
        return RenderResult(img, {k: getattr(st, k) for k, _ in abi.VkbStats._fields_})

    def set_params(self, mlp=None, table=None):
        m = None if mlp is None else np.ascontiguousarray(mlp, np.float32)
        t = None if table is None else np.ascontiguousarray(table, np.float32).reshape(-1)
        abi.check(self.r.lib.vkb_debug_nrc_set_params(self.h, abi.fptr(m) if m is not None else None, abi.fptr(t) if t is not None else None))

    def params(self, table=True):
        m = np.empty(abi.NRC_MLP_PARAMS, np.float32)
        t = np.empty(abi.NRC_HASH_PARAMS, np.float32) if table else None
        abi.check(self.r.lib.vkb_debug_nrc_get_params(self.h, abi.fptr(m), abi.fptr(t) if table else None))
        return m, t

    def forward(self, records):
        rec = np.ascontiguousarray(records, np.float32)
        n = rec.shape[0]
        x = np.empty((n, 64), np.float32); y = np.empty((n, 3), np.float32)
        abi.check(self.r.lib.vkb_debug_nrc_forward(self.h, n, abi.fptr(rec), abi.fptr(x), abi.fptr(y)))
        return x, y

    def gradients(self, records, targets, table=True):
        rec = np.ascontiguousarray(records, np.float32); tg = np.ascontiguousarray(targets, np.float32)
        g = np.empty(abi.NRC_MLP_PARAMS, np.float32)
        hg = np.empty(abi.NRC_HASH_PARAMS, np.float32) if table else None
        loss = C.c_float()
        abi.check(self.r.lib.vkb_debug_nrc_gradients(self.h, rec.shape[0], abi.fptr(rec), abi.fptr(tg), abi.fptr(g),
                                                     abi.fptr(hg) if table else None, C.byref(loss)))
        return float(loss.value), g, hg

    def step(self, records, targets) -> float:
        rec = np.ascontiguousarray(records, np.float32); tg = np.ascontiguousarray(targets, np.float32)
        loss = C.c_float()
        abi.check(self.r.lib.vkb_debug_nrc_step(self.h, rec.shape[0], abi.fptr(rec), abi.fptr(tg), C.byref(loss)))
        return float(loss.value)


def render(scene: Scene, profile: Profile | None = None, device: int = 0) -> RenderResult:
    """Render `scene` under `profile` on one GPU and return the linear mean image."""
    with Renderer(device) as r, r.install(scene) as s:
        return s.render(profile or Profile())
