"""Image environment (path.slang:961-992,1096-1120,1463; environment_proposal.slang;
environment.rs:573-620) on the GPU against the oracle, through the C ABI."""
import numpy as np
import pytest

from vork_b200 import Profile, scene as S
from vork_b200.serving import Server

pytestmark = pytest.mark.gpu


def _plane_scene(img, width=32, height=32):
    g = S.grid((200.0, 200.0), (2, 2))
    m = S.material((1, 1, 1), 0.5, 0.0)
    m.specular_weight = 0.0
    cam = S.look_at((0, 5, 0.001), (0, 0, 0), width=width, height=height, fov_y_degrees=20)
    return S.Scene([g], S.rows_from(1.0, (0, 0, 0))[None], np.zeros(1, np.uint32), np.zeros(1, np.uint32), [m], [], cam,
                   S.environment((0.0, 0.0, 0.0)), env_image=S.EnvironmentImage(img))


def _spheres_under_sky(rotation=None, width=96, height=96):
    sc = S.spheres_scene(num_spheres=24, seed=4, width=width, height=height, grid_cells=16)
    sc.environment = S.environment((0.05, 0.05, 0.05))
    kw = {} if rotation is None else {"rotation": rotation}
    sc.env_image = S.EnvironmentImage(S.sky_image(128, 64, sun_radiance=60.0), strength=0.8, color=(1.0, 0.95, 0.9), **kw)
    return sc


def test_white_plane_under_the_image_returns_its_irradiance(renderer, oracle):
    img = S.sky_image(64, 32, sun_radiance=50.0)
    sc = _plane_scene(img)
    o = oracle.OracleScene(sc)
    th = (np.arange(192) + 0.5) / 192 * np.pi
    ph = (np.arange(384) + 0.5) / 384 * 2 * np.pi
    T, PH = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.sin(T) * np.cos(PH), np.cos(T), np.sin(T) * np.sin(PH)], -1).reshape(-1, 3).astype(np.float32)
    w = (np.sin(T) * (np.pi / 192) * (2 * np.pi / 384)).reshape(-1)
    _, rq = o.env_eval(d)
    up = d[:, 1] > 0
    expected = (rq[up] * (d[up, 1] * w[up])[:, None]).sum(0) / np.pi
    with renderer.install(sc) as s:
        res = s.render(Profile.reference_transport(2, 256))
    got = res.image[..., :3].mean((0, 1))
    print("white plane under the image: GPU", got.tolist(), "expected", expected.tolist())
    assert np.allclose(got, expected, rtol=5e-3), (got, expected)
    assert res.stats["shadow_rays"] > 0 and res.stats["traversal_overflows"] == 0


@pytest.mark.parametrize("rotated", [False, True])
def test_spheres_under_the_image_match_fp32_oracle(renderer, oracle, rotated):
    c, s_ = np.cos(1.1), np.sin(1.1)
    rot = np.array([[c, 0, -s_], [0, 1, 0], [s_, 0, c]]) if rotated else None
    sc = _spheres_under_sky(rot)
    o = oracle.OracleScene(sc, fp32=True, fp64=False)
    lut = renderer.brdf_lut()
    fracs = []
    with renderer.install(sc) as s:
        for k in range(2):
            prof = Profile.reference_transport(4, 16, first_sample=k, sample_count=1)
            img = s.render(prof).image
            with oracle.atlas(lut):
                ref, _ = o.render(prof.c(), fp64=False)
            rel = np.abs(img[..., :3] - ref[..., :3]).sum(-1) / (ref[..., :3].sum(-1) + 1e-3)
            fracs.append(float(np.mean(rel < 1e-4)))
        prof = Profile.reference_transport(4, 16, sample_count=8)
        img = s.render(prof).image
    with oracle.atlas(lut):
        ref, st = o.render(prof.c(), fp64=False)
    m, mr = img[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
    print("spheres under the image: single samples within 1e-4 of the FP32 oracle", fracs, "mean ratio", (m / mr).tolist())
    assert np.all(np.abs(m / mr - 1) < 0.01), (m, mr)
    assert min(fracs) > 0.95, fracs


def test_image_scenes_in_batches_forks_and_the_server_equal_alone(renderer):
    env_scene = _spheres_under_sky(width=64, height=48)
    plain = S.spheres_scene(num_spheres=6, seed=9, width=48, height=48, grid_cells=8)
    prof = Profile.reference_transport(4, 6)
    with renderer.install(env_scene) as a, renderer.install(plain) as b:
        alone_a, alone_b = a.render(prof).image, b.render(prof).image
        imgs, _ = renderer.render_batch([(a, prof), (b, prof)], flags=4)
        assert np.array_equal(imgs[0], alone_a) and np.array_equal(imgs[1], alone_b)
        f = a.fork()
        try:
            assert np.array_equal(f.render(prof).image, alone_a)
        finally:
            f.close()
        with Server(renderer, max_jobs=4, wave_capacity=20000) as srv:
            ids = [srv.submit(b, prof), srv.submit(a, prof)]
            srv.run_until_idle()
            assert np.array_equal(srv.images[ids[0]], alone_b) and np.array_equal(srv.images[ids[1]], alone_a)
