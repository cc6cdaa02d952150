"""Emissive meshes (emitters.rs:22-44, emitter_weights.slang, emitter_mesh_proposal.slang,
path.slang:996-1002,1121-1167,1580-1591) on the GPU against the oracle, through the C ABI."""
import numpy as np
import pytest

from vork_b200 import Profile, scene as S
from vork_b200.serving import Server
from test_mesh_emitters_oracle import _lamp_over_plane, lamp_form_factor

pytestmark = pytest.mark.gpu


def test_white_plane_under_a_lamp_returns_its_form_factor(renderer):
    sc = _lamp_over_plane(width=32, height=32)
    with renderer.install(sc) as s:
        res = s.render(Profile.reference_transport(2, 256))
    expected = lamp_form_factor() * 10.0 * np.array([1.0, 0.8, 0.6])
    got = res.image[..., :3].mean((0, 1))
    print("white plane under a lamp: GPU", got.tolist(), "expected", expected.tolist())
    assert np.allclose(got, expected, rtol=5e-3), (got, expected)
    assert res.stats["shadow_rays"] > 0 and res.stats["traversal_overflows"] == 0


def _lamps(mixed):
    sc = S.lamp_scene(width=96, height=72, seed=2)
    if mixed:
        # Every strategy at once: an analytic sun, the image environment and the lamps.
        sc.lights = [S.sun_light((0.3, -1.0, 0.2), energy=2.0)]
        sc.environment = S.environment((0.02, 0.02, 0.03))
        sc.env_image = S.EnvironmentImage(S.sky_image(64, 32, sun_radiance=20.0), strength=0.5)
    return sc


@pytest.mark.parametrize("mixed", [False, True])
def test_lamp_scene_matches_fp32_oracle(renderer, oracle, mixed):
    sc = _lamps(mixed)
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
        ref, _ = o.render(prof.c(), fp64=False)
    m, mr = img[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
    print("lamps", "mixed" if mixed else "alone", ": single samples within 1e-4 of the FP32 oracle", fracs, "mean ratio", (m / mr).tolist())
    assert np.all(np.abs(m / mr - 1) < 0.01), (m, mr)
    assert min(fracs) > 0.95, fracs


def test_overlapped_waves_of_a_lamp_scene_equal_serial_waves(renderer):
    from vork_b200 import abi
    sc = S.lamp_scene(width=64, height=48, seed=8)
    sc.env_image = S.EnvironmentImage(S.sky_image(32, 16, sun_radiance=10.0), strength=0.3)
    with renderer.install(sc) as s:
        a = s.render(Profile.reference_transport(4, 6, wave_samples=1)).image
        b = s.render(Profile.reference_transport(4, 6, wave_samples=1, flags=abi.PROFILE_SERIAL_WAVES)).image
    assert np.array_equal(a, b)


def test_weight_tree_follows_instance_updates(renderer):
    # Moving and scaling the lamps (a TLAS rebuild) re-derives the weight tree: the render
    # equals a fresh install of the moved scene.
    sc = S.lamp_scene(width=48, height=36, seed=5)
    rows = sc.instance_rows.copy()
    moved = rows.copy()
    moved[1:4, :, 3] += np.array([0.5, 0.3, -0.4], np.float32)
    moved[1:4, 0, 0] *= 1.5
    prof = Profile.reference_transport(4, 4)
    with renderer.install(sc) as a:
        a.update_instances(moved, policy=1)
        updated = a.render(prof).image
    sc.instance_rows = moved
    with renderer.install(sc) as b:
        fresh = b.render(prof).image
    assert np.array_equal(updated, fresh)


def test_lamp_scenes_in_batches_forks_and_the_server_equal_alone(renderer):
    lamps = S.lamp_scene(width=64, height=48, seed=7)
    plain = S.spheres_scene(num_spheres=6, seed=9, width=48, height=48, grid_cells=8)
    prof = Profile.reference_transport(4, 6)
    with renderer.install(lamps) as a, renderer.install(plain) as b:
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
