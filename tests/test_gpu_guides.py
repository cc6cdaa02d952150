"""Denoiser guide planes (path.slang:1549-1571 per sample, summed as path.slang:1956-1963)
against the oracle's restatement, through the C ABI."""
import ctypes as C

import numpy as np
import pytest

from vork_b200 import Profile, abi, scene as S

pytestmark = pytest.mark.gpu


def test_white_diffuse_plane_guides_are_its_colour_and_normal(renderer):
    # Specular weight 0: the dielectric interface vanishes (ior 1), so the response to a
    # uniform white world is the base colour itself and nothing is reflected.
    g = S.grid((200.0, 200.0), (2, 2))
    m = S.material((0.8, 0.6, 0.4), 0.5, 0.0)
    m.specular_weight = 0.0
    cam = S.look_at((0, 5, 0.001), (0, 0, 0), width=32, height=32, fov_y_degrees=30)
    sc = S.Scene([g], S.rows_from(1.0, (0, 0, 0))[None], np.zeros(1, np.uint32), np.zeros(1, np.uint32), [m], [], cam,
                 S.environment((1.0, 0.75, 0.5)))
    with renderer.install(sc) as s:
        res = s.render(Profile.reference_transport(4, 8), guides=True)
    assert np.allclose(res.guide_albedo.reshape(-1, 4), [0.8, 0.6, 0.4, 1.0], rtol=1e-5, atol=1e-6)
    assert np.allclose(res.guide_normal.reshape(-1, 4), [0.0, 1.0, 0.0, 0.0], atol=1e-5)


def test_guides_match_the_oracle_and_leave_the_image_alone(renderer, oracle, small_scene):
    prof = Profile.reference_transport(4, 16, sample_count=4)
    o = oracle.OracleScene(small_scene, fp32=True, fp64=False)
    with renderer.install(small_scene) as s:
        res = s.render(prof, guides=True)
        plain = s.render(prof)
    assert np.array_equal(res.image, plain.image)            # guides are a side output
    with oracle.atlas(renderer.brdf_lut()):
        _, _, g = o.render(prof.c(), fp64=False, guides=True)
    ga, gn = g[:, :, 0], g[:, :, 1]
    # Coverage: the samples' camera hits; a pixel differs only where a sample's primary hit
    # differs (a shared edge or silhouette).
    da = np.abs(res.guide_albedo - ga).max(-1)
    dn = np.abs(res.guide_normal - gn).max(-1)
    print("guides vs FP32 oracle: pixels within 1e-4 (albedo, normal):", float(np.mean(da < 1e-4)), float(np.mean(dn < 1e-4)))
    assert np.mean(da < 1e-4) > 0.995 and np.mean(dn < 1e-4) > 0.995
    assert np.allclose(res.guide_albedo.mean((0, 1)), ga.mean((0, 1)), rtol=1e-3, atol=1e-5)
    cov = res.guide_albedo[..., 3]
    assert 0.2 < cov.mean() < 1.0 and np.all((cov >= 0) & (cov <= 1))
    assert np.all(res.guide_albedo[..., :3] <= 1.0 + 1e-6) and np.all(res.guide_albedo[..., :3] >= 0.0)
    n = np.linalg.norm(res.guide_normal[..., :3], axis=-1)
    assert np.all(n <= 1.0 + 1e-5)


def test_guides_are_refused_outside_single_plain_renders(renderer, small_scene):
    with renderer.install(small_scene) as s:
        with pytest.raises(abi.VkbError) as e:
            s.render(Profile(samples=16, adaptive=True), guides=True)
        assert e.value.status == abi.VKB_UNSUPPORTED
        # Two jobs of a batch asking for guides.
        ga = np.empty((256, 256, 4), np.float32)
        jobs = (abi.VkbJob * 2)()
        imgs = [np.empty((256, 256, 4), np.float32) for _ in range(2)]
        for k in range(2):
            jobs[k].scene = s.h
            jobs[k].profile = Profile.reference_transport(4, 2).c()
            jobs[k].out.rgba = imgs[k].ctypes.data_as(C.c_void_p)
            jobs[k].out.guide_albedo = ga.ctypes.data_as(C.c_void_p)
        st = abi.VkbStats()
        assert renderer.lib.vkb_render_batch(renderer.h, jobs, 2, 0, C.byref(st)) == abi.VKB_UNSUPPORTED
