"""ctypes mirror of include/vkb.h and the loader of the in-tree CUDA library.

The product path is the CUDA library ``vork_b200/_lib/libvkb.so`` built for sm_100a;
there is no CPU fallback: ``load()`` raises when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_DIR = Path(__file__).resolve().parent / "_lib"
LIB_PATH = LIB_DIR / "libvkb.so"

VKB_OK, VKB_INVALID_ARG, VKB_OUT_OF_MEMORY, VKB_DEVICE_TIMEOUT, VKB_NONFINITE, VKB_INTERNAL, VKB_UNSUPPORTED = range(7)
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OUT_OF_MEMORY", 3: "DEVICE_TIMEOUT", 4: "NONFINITE", 5: "INTERNAL", 6: "UNSUPPORTED"}

RAY_CAMERA, RAY_SHADOW, RAY_DIFFUSE, RAY_SPECULAR, RAY_TRANSMISSION, RAY_VOLUME = 1, 2, 4, 8, 16, 32
LIGHT_LINK_ALL = 64
LIGHT_RAY_SHADOWED, LIGHT_RAY_SHADOWED_BY_ALL = 1, 2


class VkbMesh(C.Structure):
    _fields_ = [("positions", C.POINTER(C.c_float)), ("normals", C.POINTER(C.c_float)),
                ("indices", C.POINTER(C.c_uint32)), ("num_vertices", C.c_uint32), ("num_triangles", C.c_uint32)]


class VkbMaterial(C.Structure):
    _fields_ = [("base_weight", C.c_float), ("base_color", C.c_float * 3), ("base_metalness", C.c_float),
                ("specular_weight", C.c_float), ("specular_color", C.c_float * 3), ("specular_roughness", C.c_float),
                ("specular_ior", C.c_float), ("emission_luminance", C.c_float), ("emission_color", C.c_float * 3),
                ("flags", C.c_uint32)]


class VkbLight(C.Structure):
    _fields_ = [("shadow_offsets", C.c_uint32 * 8), ("position", C.c_float * 4), ("direction", C.c_float * 4),
                ("radiance", C.c_float * 4), ("params", C.c_float * 4), ("emitter_u", C.c_float * 4),
                ("emitter_v", C.c_float * 4), ("emission", C.c_float * 4), ("projection", C.c_float * 4)]


class VkbCamera(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("right", C.c_float * 3), ("up", C.c_float * 3), ("forward", C.c_float * 3),
                ("proj_x", C.c_float), ("proj_y", C.c_float), ("near_plane", C.c_float), ("far_plane", C.c_float),
                ("width", C.c_uint32), ("height", C.c_uint32)]


class VkbEnvironment(C.Structure):
    _fields_ = [("radiance", C.c_float * 3), ("exposure", C.c_float), ("background", C.c_float * 3),
                ("camera_sees_environment", C.c_uint32)]


class VkbEnvironmentImage(C.Structure):
    _fields_ = [("rgba", C.POINTER(C.c_float)), ("width", C.c_uint32), ("height", C.c_uint32), ("strength", C.c_float),
                ("color", C.c_float * 3), ("rotation", C.c_float * 9)]


class VkbSceneDesc(C.Structure):
    _fields_ = [("meshes", C.POINTER(VkbMesh)), ("num_meshes", C.c_uint32), ("num_instances", C.c_uint32),
                ("instance_rows", C.POINTER(C.c_float)), ("instance_mesh", C.POINTER(C.c_uint32)),
                ("instance_material", C.POINTER(C.c_uint32)), ("materials", C.POINTER(VkbMaterial)),
                ("num_materials", C.c_uint32), ("lights", C.POINTER(VkbLight)), ("num_lights", C.c_uint32),
                ("camera", VkbCamera), ("environment", VkbEnvironment), ("tlas_builder", C.c_uint32),
                ("environment_image", C.POINTER(VkbEnvironmentImage)), ("blas_format", C.c_uint32),
                ("blas_builder", C.c_uint32)]


class VkbProfile(C.Structure):
    _fields_ = [("samples", C.c_uint32), ("first_sample", C.c_uint32), ("sample_count", C.c_uint32), ("seed", C.c_uint32),
                ("bounces", C.c_uint32 * 4), ("transparent", C.c_uint32), ("caustics", C.c_uint32),
                ("clamp_direct", C.c_float), ("clamp_indirect", C.c_float), ("light_threshold", C.c_float),
                ("adaptive", C.c_uint32), ("wave_samples", C.c_uint32), ("flags", C.c_uint32),
                ("adaptive_threshold", C.c_float), ("adaptive_min_samples", C.c_uint32)]


class VkbCacheConfig(C.Structure):
    _fields_ = [("train_records", C.c_uint32), ("train_steps", C.c_uint32), ("query_vertex", C.c_uint32), ("seed", C.c_uint32),
                ("lr_mlp", C.c_float), ("lr_hash", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float)]


class VkbCacheStats(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("records", C.c_uint64), ("loss", C.c_float), ("train_ms", C.c_float),
                ("paths_ms", C.c_float), ("steps_ms", C.c_float), ("host_ms", C.c_float)]


NRC_MLP_PARAMS, NRC_HASH_PARAMS = 17408, 16777216
DISPLAY_SRGB, DISPLAY_P3, DISPLAY_REC2100_PQ, DISPLAY_REC2100_HLG = 0, 1, 2, 3


class VkbDisplayParams(C.Structure):
    _fields_ = [("display", C.c_uint32), ("exposure", C.c_float), ("gamma", C.c_float), ("peak_luminance", C.c_float),
                ("reference_white", C.c_float), ("bits", C.c_uint32), ("unassociate", C.c_uint32), ("reserved", C.c_uint32)]
PROFILE_TIME_KERNELS, PROFILE_COUNT_TRAVERSAL, PROFILE_SERIAL_WAVES = 1, 2, 16
BATCH_FAIR, BATCH_PACKED = 4, 8
TLAS_LBVH, TLAS_PLOC = 0, 1
BLAS_WIDE4, BLAS_WIDE8 = 0, 1
BLAS_BUILD_SAH, BLAS_BUILD_LBVH, BLAS_BUILD_PLOC = 0, 1, 2
NOALLOC_SCRATCH_MIB = 32


class VkbOutput(C.Structure):
    _fields_ = [("rgba", C.c_void_p), ("on_device", C.c_uint32), ("primary_ids", C.POINTER(C.c_uint32)),
                ("guide_albedo", C.c_void_p), ("guide_normal", C.c_void_p)]


class VkbStats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("dropped_path_samples", C.c_uint64), ("dropped_light_samples", C.c_uint64),
                ("traversal_overflows", C.c_uint64), ("render_ms", C.c_float), ("build_ms", C.c_float),
                ("trace_ms", C.c_float), ("trace_launches", C.c_uint32), ("kernel_launches", C.c_uint32),
                ("nodes_visited", C.c_uint64), ("triangles_tested", C.c_uint64), ("instances_entered", C.c_uint64),
                ("shadow_nodes_visited", C.c_uint64), ("shadow_triangles_tested", C.c_uint64),
                ("blas_nodes_visited", C.c_uint64), ("cache_ms", C.c_float), ("cache_queries", C.c_uint64),
                ("samples_skipped", C.c_uint64)]


class VkbJob(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("profile", VkbProfile), ("out", VkbOutput)]


class VkbTuneResult(C.Structure):
    _fields_ = [("tried", C.c_uint32), ("best_blocks_per_sm", C.c_uint32), ("best_capacity", C.c_uint64), ("best_ms", C.c_float),
                ("blocks_per_sm", C.c_uint32 * 16), ("capacity", C.c_uint64 * 16), ("ms", C.c_float * 16)]


class VkbServerConfig(C.Structure):
    _fields_ = [("memory_budget_bytes", C.c_uint64), ("max_jobs", C.c_uint32), ("flags", C.c_uint32), ("wave_capacity", C.c_uint64),
                ("aging_paths_per_s", C.c_double)]


class VkbServerStatus(C.Structure):
    _fields_ = [("queued", C.c_uint32), ("running", C.c_uint32), ("finished", C.c_uint32), ("reserved", C.c_uint32),
                ("used_bytes", C.c_uint64), ("peak_bytes", C.c_uint64)]


class VkbSceneInfo(C.Structure):
    _fields_ = [("num_instances", C.c_uint64), ("num_triangles", C.c_uint64), ("scene_bytes", C.c_uint64),
                ("tlas_rebuilds", C.c_uint64), ("tlas_refits", C.c_uint64), ("motion_bytes", C.c_uint64),
                ("build_ms", C.c_float), ("reserved", C.c_uint32), ("install_ms", C.c_float), ("blas_host_ms", C.c_float),
                ("upload_ms", C.c_float), ("tlas_ms", C.c_float)]


# Every symbol include/vkb.h declares, with its ctypes signature.
_P = C.c_void_p
SIGNATURES = {
    "vkb_abi_version": (C.c_uint32, []),
    "vkb_last_error": (C.c_char_p, []),
    "vkb_open": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "vkb_close": (C.c_int, [_P]),
    "vkb_scene_create": (C.c_int, [_P, C.POINTER(VkbSceneDesc), C.POINTER(_P)]),
    "vkb_scene_destroy": (C.c_int, [_P]),
    "vkb_scene_update_instances": (C.c_int, [_P, C.POINTER(C.c_float), C.c_uint32, C.c_int]),
    "vkb_scene_update_instances_device": (C.c_int, [_P, C.c_void_p, C.c_uint32, C.c_int]),
    "vkb_render": (C.c_int, [_P, C.POINTER(VkbProfile), C.POINTER(VkbOutput), C.POINTER(VkbStats)]),
    "vkb_render_noalloc": (C.c_int, [_P, C.POINTER(VkbProfile), C.POINTER(VkbOutput), C.POINTER(VkbStats)]),
    "vkb_render_view": (C.c_int, [_P, C.c_void_p, C.POINTER(VkbProfile), C.POINTER(VkbOutput), C.POINTER(VkbStats)]),
    "vkb_scene_fork": (C.c_int, [_P, C.POINTER(_P)]),
    "vkb_server_submit_view": (C.c_int, [_P, _P, C.c_void_p, C.POINTER(VkbProfile), C.POINTER(C.c_float), C.POINTER(C.c_uint64)]),
    "vkb_scene_info": (C.c_int, [_P, C.POINTER(VkbSceneInfo)]),
    "vkb_server_create": (C.c_int, [_P, C.POINTER(VkbServerConfig), C.POINTER(_P)]),
    "vkb_server_submit": (C.c_int, [_P, _P, C.POINTER(VkbProfile), C.POINTER(C.c_float), C.POINTER(C.c_uint64)]),
    "vkb_server_step": (C.c_int, [_P, C.POINTER(VkbServerStatus)]),
    "vkb_server_poll": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_int)]),
    "vkb_server_destroy": (C.c_int, [_P]),
    "vkb_render_batch": (C.c_int, [_P, C.POINTER(VkbJob), C.c_uint32, C.c_uint32, C.POINTER(VkbStats)]),
    "vkb_autotune": (C.c_int, [_P, C.POINTER(VkbJob), C.c_uint32, C.POINTER(VkbTuneResult)]),
    "vkb_ctx_stream": (C.c_void_p, [_P]),
    "vkb_scene_launch_count": (C.c_uint64, [_P]),
    "vkb_debug_sampler_groups": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                           C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_uint32, C.c_uint32,
                                           C.POINTER(C.c_uint32)]),
    "vkb_debug_brdf_lut": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "vkb_debug_tlas_morton": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "vkb_debug_blas_morton": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "vkb_debug_trace": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_float)]),
    "vkb_debug_occluded": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_uint32)]),
    "vkb_debug_tlas_stats": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "vkb_display": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, C.c_uint32, C.c_void_p, C.c_int]),
    "vkb_cache_create": (C.c_int, [_P, C.c_void_p, C.POINTER(_P)]),
    "vkb_cache_destroy": (C.c_int, [_P]),
    "vkb_cache_train": (C.c_int, [_P, C.POINTER(VkbProfile), C.c_void_p]),
    "vkb_render_cached": (C.c_int, [_P, C.POINTER(VkbProfile), C.POINTER(VkbOutput), C.POINTER(VkbStats)]),
    "vkb_debug_nrc_set_params": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "vkb_debug_nrc_get_params": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "vkb_debug_nrc_forward": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "vkb_debug_nrc_gradients": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                          C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "vkb_debug_nrc_step": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
}

_lib = None


class VkbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"vkb {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load(path: os.PathLike | str | None = None) -> C.CDLL:
    """Load the CUDA library (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: build it with `python -m vork_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status: int) -> None:
    if status != VKB_OK:
        msg = load().vkb_last_error()
        raise VkbError(status, msg.decode() if msg else "")


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


def uptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_uint32))
