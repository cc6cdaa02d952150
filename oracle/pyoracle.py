"""ORACLE (test infrastructure): ctypes wrapper of oracle/_build/liboracle.so.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import this.
The library is the CPU restatement of the reference's path math (oracle/oracle.cpp).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < (HERE / "oracle.cpp").stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"], check=True, capture_output=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        l = C.CDLL(str(LIB))
        P = C.c_void_p
        u32p, f32p, f64p = C.POINTER(C.c_uint32), C.POINTER(C.c_float), C.POINTER(C.c_double)
        l.oracle_sampler_bits.argtypes = [C.c_uint32, u32p, u32p, u32p, u32p, C.c_uint32, C.c_uint32, u32p, C.c_int]
        l.oracle_sobol_directions.argtypes = [u32p]
        l.oracle_sobol_points.argtypes = [C.c_uint32, u32p]
        l.oracle_filter_table.argtypes = [f32p]
        l.oracle_filter_cdf.argtypes = [C.c_double]
        l.oracle_filter_cdf.restype = C.c_double
        l.oracle_brdf_lut.argtypes = [C.c_int, f32p]
        l.oracle_half_round.argtypes = [C.c_float]
        l.oracle_half_round.restype = C.c_float
        l.oracle_emitter_sample.argtypes = [P, f64p, f64p, f64p, f64p, f64p, f64p]
        l.oracle_emitter_eval.argtypes = [P, f64p, f64p, f64p, f64p, f64p]
        l.oracle_bsdf.argtypes = [P, f64p, f64p, f64p, f64p, f64p, u32p]
        l.oracle_scene_create.argtypes = [P, C.c_int]
        l.oracle_scene_create.restype = P
        l.oracle_scene_destroy.argtypes = [P]
        l.oracle_trace.argtypes = [P, C.c_int, C.c_uint32, f32p, C.c_int, f32p, u32p, f32p]
        l.oracle_camera_rays.argtypes = [P, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, f32p]
        l.oracle_render.argtypes = [P, C.c_int, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, f32p, u32p, C.c_uint32,
                                    C.POINTER(C.c_uint64), f32p]
        l.oracle_tlas_morton.argtypes = [P, u32p]
        l.oracle_instance_boxes.argtypes = [P, f32p, f32p]
        l.oracle_blas_morton.argtypes = [P, C.c_uint32, u32p]
        l.oracle_set_lut.argtypes = [f32p]
        l.oracle_env_sample.argtypes = [P, C.c_int, C.c_uint32, f32p, f32p, f32p]
        l.oracle_env_eval.argtypes = [P, C.c_uint32, f32p, f32p, f32p]
        l.oracle_mesh_tree.argtypes = [P, f32p]
        l.oracle_mesh_tree.restype = C.c_uint32
        l.oracle_mesh_triangles.argtypes = [P]
        l.oracle_mesh_triangles.restype = C.c_uint32
        l.oracle_mesh_sample.argtypes = [P, C.c_uint32, f32p, u32p, u32p, f32p, f32p]
        l.oracle_mesh_probability.argtypes = [P, C.c_uint32, u32p, u32p, f32p]
        _lib = l
    return _lib


def _u(a):
    return np.ascontiguousarray(a, np.uint32)


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def sampler_bits(px, py, index, groups, count, stream, mode=0):
    px, py, index, groups = _u(px), _u(py), _u(index), _u(groups)
    out = np.zeros((px.size, 4), np.uint32)
    lib().oracle_sampler_bits(px.size, _p(px, C.c_uint32), _p(py, C.c_uint32), _p(index, C.c_uint32), _p(groups, C.c_uint32),
                              count, stream, _p(out, C.c_uint32), mode)
    return out


def sobol_directions():
    out = np.zeros((3, 32), np.uint32)
    lib().oracle_sobol_directions(_p(out, C.c_uint32))
    return out


def sobol_points(n):
    out = np.zeros((n, 4), np.uint32)
    lib().oracle_sobol_points(n, _p(out, C.c_uint32))
    return out


def filter_table():
    out = np.zeros(1025, np.float32)
    lib().oracle_filter_table(_p(out, C.c_float))
    return out


def brdf_lut(fp64=False):
    out = np.zeros((2240, 128, 4), np.float32)
    lib().oracle_brdf_lut(1 if fp64 else 0, _p(out, C.c_float))
    return out


class atlas:
    """Within the block the oracle reads `texels` ((2240, 128, 4) float32, e.g. the
    device-baked atlas) instead of its own bake, so a transport comparison measures the
    transport alone; the bake itself is compared on its own."""

    def __init__(self, texels):
        self.texels = np.ascontiguousarray(texels, np.float32)
        assert self.texels.shape == (2240, 128, 4)

    def __enter__(self):
        lib().oracle_set_lut(_p(self.texels, C.c_float))
        return self

    def __exit__(self, *exc):
        lib().oracle_set_lut(None)


def emitter_sample(light, world, u):
    w = np.asarray(world, np.float64); uu = np.asarray(u, np.float64)
    d = np.zeros(3); r = np.zeros(3); pdf = C.c_double(); dist = C.c_double()
    lib().oracle_emitter_sample(C.byref(light), _p(w, C.c_double), _p(uu, C.c_double), _p(d, C.c_double), _p(r, C.c_double),
                                C.byref(pdf), C.byref(dist))
    return d, r, pdf.value, dist.value


def emitter_eval(light, world, direction):
    w = np.asarray(world, np.float64); dd = np.asarray(direction, np.float64)
    r = np.zeros(3); pdf = C.c_double(); dist = C.c_double()
    lib().oracle_emitter_eval(C.byref(light), _p(w, C.c_double), _p(dd, C.c_double), _p(r, C.c_double), C.byref(pdf), C.byref(dist))
    return r, pdf.value, dist.value


def bsdf_sample(material, view, u3):
    v = np.asarray(view, np.float64); u = np.asarray(u3, np.float64)
    d = np.zeros(3); w = np.zeros(3); pdf = C.c_double(); ev = C.c_uint32()
    lib().oracle_bsdf(C.byref(material), _p(v, C.c_double), _p(u, C.c_double), _p(d, C.c_double), _p(w, C.c_double),
                      C.byref(pdf), C.byref(ev))
    return d, w, pdf.value, ev.value


class OracleScene:
    """The oracle's copy of a scene (FP32 and FP64 restatements)."""

    def __init__(self, scene, fp32=True, fp64=True):
        self.scene = scene
        self.desc = scene.desc()
        self.h = lib().oracle_scene_create(C.byref(self.desc), (1 if fp32 else 0) | (2 if fp64 else 0))

    def close(self):
        if self.h:
            lib().oracle_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def trace(self, rays7: np.ndarray, fp64=True, any_hit=False, threads=None):
        """Closest (or any) hits of (origin, dir, tmax) rays, in chunks over host threads."""
        from concurrent.futures import ThreadPoolExecutor
        r = np.ascontiguousarray(rays7, np.float32)
        n = r.shape[0]
        t = np.zeros(n, np.float32); ids = np.zeros((n, 2), np.uint32); uv = np.zeros((n, 2), np.float32)

        def chunk(a, b):
            lib().oracle_trace(self.h, 1 if fp64 else 0, b - a, _p(r[a:b], C.c_float), 1 if any_hit else 0, _p(t[a:b], C.c_float),
                               _p(ids[a:b], C.c_uint32), _p(uv[a:b], C.c_float))
        threads = threads or os.cpu_count() or 1
        step = max(1024, -(-n // (4 * threads)))
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(lambda a: chunk(a, min(n, a + step)), range(0, n, step)))
        return t, ids, uv

    def env_sample(self, u2, fp64=True):
        """Proposal samples of the image environment: (directions (n,3), pdfs (n,))."""
        u = np.ascontiguousarray(u2, np.float32).reshape(-1, 2)
        d = np.zeros((len(u), 3), np.float32); p = np.zeros(len(u), np.float32)
        lib().oracle_env_sample(self.h, 1 if fp64 else 0, len(u), _p(u, C.c_float), _p(d, C.c_float), _p(p, C.c_float))
        return d, p

    def env_eval(self, dirs):
        """(proposal pdf, radiance) of world directions under the image environment."""
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        p = np.zeros(len(d), np.float32); rgb = np.zeros((len(d), 3), np.float32)
        lib().oracle_env_eval(self.h, len(d), _p(d, C.c_float), _p(p, C.c_float), _p(rgb, C.c_float))
        return p, rgb

    def mesh_tree(self):
        """The emissive-mesh weight tree (2 x leaves floats, node 1 the root) and its leaf count."""
        leaves = lib().oracle_mesh_tree(self.h, None)
        out = np.zeros(2 * leaves, np.float32)
        if leaves:
            lib().oracle_mesh_tree(self.h, _p(out, C.c_float))
        return out, leaves

    def mesh_triangles(self):
        return int(lib().oracle_mesh_triangles(self.h))

    def mesh_sample(self, u3):
        """Source samples for uniforms u (n,3): (instance, primitive, barycentrics (n,2), probability)."""
        u = np.ascontiguousarray(u3, np.float32).reshape(-1, 3)
        n = len(u)
        inst = np.zeros(n, np.uint32); prim = np.zeros(n, np.uint32); b = np.zeros((n, 2), np.float32); pr = np.zeros(n, np.float32)
        lib().oracle_mesh_sample(self.h, n, _p(u, C.c_float), _p(inst, C.c_uint32), _p(prim, C.c_uint32), _p(b, C.c_float), _p(pr, C.c_float))
        return inst, prim, b, pr

    def mesh_probability(self, inst, prim):
        i = np.ascontiguousarray(inst, np.uint32); q = np.ascontiguousarray(prim, np.uint32)
        out = np.zeros(len(i), np.float32)
        lib().oracle_mesh_probability(self.h, len(i), _p(i, C.c_uint32), _p(q, C.c_uint32), _p(out, C.c_float))
        return out

    def camera_rays(self, profile, index, x0=0, y0=0, w=None, h=None):
        cam = self.scene.camera
        w = cam.width if w is None else w
        h = cam.height if h is None else h
        out = np.zeros((h * w, 7), np.float32)
        lib().oracle_camera_rays(self.h, C.cast(C.byref(profile), C.c_void_p), index, x0, y0, w, h, _p(out, C.c_float))
        return out

    def render(self, profile, x0=0, y0=0, w=None, h=None, fp64=True, threads=None, ids=False, guides=False):
        """(image, stats), or (image, ids, stats) with ids; with guides=True also the
        (h, w, 2, 4) guide planes (mean albedo + coverage, mean normal) appended."""
        cam = self.scene.camera
        w = cam.width if w is None else w
        h = cam.height if h is None else h
        if profile.adaptive and ((x0, y0, w, h) != (0, 0, cam.width, cam.height) or profile.first_sample
                                 or profile.sample_count not in (0, profile.samples)):
            raise ValueError("the adaptive oracle renders a whole image and a whole exposure")
        threads = threads or os.cpu_count() or 1
        out = np.zeros((h, w, 4), np.float32)
        idbuf = np.zeros((h, w, 2), np.uint32) if ids else None
        if guides and profile.adaptive:
            raise ValueError("guides are rendered without adaptive stopping")
        gbuf = np.zeros((h, w, 2, 4), np.float32) if guides else None
        stats = (C.c_uint64 * 4)()
        lib().oracle_render(self.h, 1 if fp64 else 0, C.cast(C.byref(profile), C.c_void_p), x0, y0, w, h, _p(out, C.c_float),
                            _p(idbuf, C.c_uint32) if ids else None, threads, stats, _p(gbuf, C.c_float) if guides else None)
        st = {"extension_rays": stats[0], "shadow_rays": stats[1], "dropped_path_samples": stats[2], "dropped_light_samples": stats[3]}
        res = (out, idbuf, st) if ids else (out, st)
        return res + (gbuf,) if guides else res

    def tlas_morton(self):
        out = np.zeros(self.desc.num_instances, np.uint32)
        lib().oracle_tlas_morton(C.cast(C.byref(self.desc), C.c_void_p), _p(out, C.c_uint32))
        return out

    def instance_boxes(self):
        """(lo, hi): the TLAS leaf world boxes, (n, 3) float32 each."""
        n = self.desc.num_instances
        lo = np.zeros((n, 3), np.float32); hi = np.zeros((n, 3), np.float32)
        lib().oracle_instance_boxes(C.cast(C.byref(self.desc), C.c_void_p), _p(lo, C.c_float), _p(hi, C.c_float))
        return lo, hi

    def blas_morton(self, mesh):
        out = np.zeros(self.scene.meshes[mesh].num_triangles, np.uint32)
        lib().oracle_blas_morton(C.cast(C.byref(self.desc), C.c_void_p), mesh, _p(out, C.c_uint32))
        return out
