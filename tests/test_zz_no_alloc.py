"""The render entry point that allocates nothing (vkb_render_noalloc), against vkb_render.

Callers such as a host renderer that owns all device memory through its own manager,
or a serving loop whose footprint is fixed after admission, cannot let the library call
cudaMalloc while they render.  vkb_render_noalloc renders from one fixed device array
instead; its results must be the ones vkb_render gives, call after call, even though
every call reuses (and must first clear) the same array.  This file is collected last
and builds its own renderer, so it passes alone in a fresh process or after the rest.
"""
import ctypes as C

import numpy as np
import pytest

from vork_b200 import Profile, Renderer, abi, scene as S

pytestmark = pytest.mark.gpu


def _noalloc(installed, profile, ids=False):
    cam = installed.scene.camera
    img = np.empty((cam.height, cam.width, 4), np.float32)
    out = abi.VkbOutput()
    out.rgba = img.ctypes.data_as(C.c_void_p)
    out.on_device = 0
    idbuf = np.empty((cam.height, cam.width, 2), np.uint32) if ids else None
    out.primary_ids = abi.uptr(idbuf) if ids else None
    st = abi.VkbStats()
    p = profile.c()
    abi.check(installed.r.lib.vkb_render_noalloc(installed.h, C.byref(p), C.byref(out), C.byref(st)))
    return img, idbuf, st


def test_noalloc_render_matches_render_on_two_calls():
    sc = S.spheres_scene(width=160, height=120)
    prof = Profile.reference_transport(4, 8)
    with Renderer(0) as r, r.install(sc) as s:
        ref = s.render(prof, ids=True)
        for _ in range(2):
            img, ids, st = _noalloc(s, prof, ids=True)
            # Same kernels, same per-sample order: bit-identical (well inside the 1e-5 tolerance).
            assert np.array_equal(img, ref.image)
            assert np.array_equal(ids, ref.primary_ids)
            assert st.paths == 160 * 120 * 8 and st.traversal_overflows == 0
        # A different sample range right after must not see stale accumulators.
        part = Profile.reference_transport(4, 8, first_sample=4, sample_count=4)
        img, _, _ = _noalloc(s, part)
        assert np.array_equal(img, s.render(part).image)


def test_noalloc_rejects_images_beyond_its_scratch():
    big = S.spheres_scene(width=1024, height=1024)
    with Renderer(0) as r, r.install(big) as s:
        with pytest.raises(abi.VkbError) as e:
            _noalloc(s, Profile.reference_transport(4, 1))
        assert e.value.status == abi.VKB_INVALID_ARG
        assert "scratch" in str(e.value)
