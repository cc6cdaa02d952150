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


def test_noalloc_allocates_nothing_on_a_fresh_renderer():
    # The property the entry point exists for: on a renderer that has never rendered
    # (so no wavefront of its own exists), a no-allocation render leaves the device's
    # free memory unchanged, and is still right.  A first renderer loads the library's
    # device code (lazy module loading allocates for code, not for the render).
    import torch
    sc = S.spheres_scene(width=128, height=96)
    prof = Profile.reference_transport(4, 16)
    with Renderer(0) as warm, warm.install(sc) as s:
        _noalloc(s, prof)
    with Renderer(0) as r, r.install(sc) as s:
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(0)
        img, _, st = _noalloc(s, prof)
        img2, _, _ = _noalloc(s, prof)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info(0)
        # vkb_render would have reserved 128 x 96 x 16 path slots (~43 MB) here.
        assert free0 - free1 < (1 << 20), (free0, free1)
        assert np.array_equal(img, img2) and st.paths == 128 * 96 * 16 and st.kernel_launches > 0
        assert np.array_equal(img, s.render(prof).image)


def test_noalloc_rejects_images_beyond_its_scratch():
    big = S.spheres_scene(width=1024, height=1024)
    with Renderer(0) as r, r.install(big) as s:
        with pytest.raises(abi.VkbError) as e:
            _noalloc(s, Profile.reference_transport(4, 1))
        assert e.value.status == abi.VKB_INVALID_ARG
        assert "scratch" in str(e.value)
