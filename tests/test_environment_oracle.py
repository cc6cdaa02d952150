"""The oracle's image environment (environment_proposal.slang, environment.rs:573-620,
path.slang:961-992,1096-1120,1463) on CPU: the proposal's pdf is the density it samples
with and integrates to one; sampling by it integrates the radiance; a white Lambert
plane under the image returns the image's cosine-weighted irradiance / pi."""
import numpy as np
import pytest

from vork_b200 import Profile, scene as S


def _plane_scene(img, rotation=None):
    g = S.grid((200.0, 200.0), (2, 2))
    m = S.material((1, 1, 1), 0.5, 0.0)
    m.specular_weight = 0.0
    cam = S.look_at((0, 5, 0.001), (0, 0, 0), width=8, height=8, fov_y_degrees=20)
    env = S.EnvironmentImage(img) if rotation is None else S.EnvironmentImage(img, rotation=rotation)
    return S.Scene([g], S.rows_from(1.0, (0, 0, 0))[None], np.zeros(1, np.uint32), np.zeros(1, np.uint32), [m], [], cam,
                   S.environment((0.0, 0.0, 0.0)), env_image=env)


def _sphere_quadrature(n_theta=192, n_phi=384):
    th = (np.arange(n_theta) + 0.5) / n_theta * np.pi
    ph = (np.arange(n_phi) + 0.5) / n_phi * 2 * np.pi
    T, PH = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.sin(T) * np.cos(PH), np.cos(T), np.sin(T) * np.sin(PH)], -1).reshape(-1, 3)
    w = (np.sin(T) * (np.pi / n_theta) * (2 * np.pi / n_phi)).reshape(-1)
    return d.astype(np.float32), w


@pytest.mark.parametrize("rotated", [False, True])
def test_proposal_density_and_sampling(oracle, rotated):
    c, s_ = np.cos(0.7), np.sin(0.7)
    rot = np.array([[c, 0, -s_], [0, 1, 0], [s_, 0, c]]) if rotated else None
    o = oracle.OracleScene(_plane_scene(S.sky_image(64, 32, sun_radiance=50.0), rot))
    u = np.random.default_rng(1).random((100000, 2)).astype(np.float32)
    d, p = o.env_sample(u)
    p2, rgb = o.env_eval(d)
    assert np.all(p > 0) and np.allclose(p, p2, rtol=1e-5)
    assert np.allclose(np.linalg.norm(d, axis=1), 1, atol=1e-5)
    dq, w = _sphere_quadrature()
    pq, rq = o.env_eval(dq)
    assert abs((pq * w).sum() - 1) < 1e-3
    quad = (rq * w[:, None]).sum(0)
    assert np.allclose((rgb / p[:, None]).mean(0), quad, rtol=2e-3), ((rgb / p[:, None]).mean(0), quad)


def test_black_image_falls_back_to_the_uniform_sphere(oracle):
    o = oracle.OracleScene(_plane_scene(np.zeros((16, 32, 4), np.float32)))
    d, p = o.env_sample(np.random.default_rng(2).random((2000, 2)).astype(np.float32))
    assert np.allclose(p, 1 / (4 * np.pi), rtol=1e-3)


def test_white_plane_under_the_image_returns_its_irradiance(oracle):
    # Environment NEE plus the MIS-weighted escapes of BSDF samples: an unbiased estimate
    # of the cosine-weighted irradiance / pi of the upper hemisphere.
    o = oracle.OracleScene(_plane_scene(S.sky_image(64, 32, sun_radiance=50.0)))
    dq, w = _sphere_quadrature()
    _, rq = o.env_eval(dq)
    up = dq[:, 1] > 0
    expected = (rq[up] * (dq[up, 1] * w[up])[:, None]).sum(0) / np.pi
    img, st = o.render(Profile.reference_transport(2, 128).c(), fp64=True)
    assert np.allclose(img[..., :3].mean((0, 1)), expected, rtol=5e-3), (img[..., :3].mean((0, 1)), expected)
    assert st["shadow_rays"] > 0
