"""CUDA path against the oracle and the reference's known answers, through the C ABI."""
import dataclasses
import json
from pathlib import Path

import numpy as np
import pytest

from vork_b200 import Profile, abi, scene as S

GOLDEN = Path(__file__).resolve().parent / "golden"
pytestmark = pytest.mark.gpu


def test_sampler_bits_match_golden_and_oracle(renderer, oracle):
    g = np.load(GOLDEN / "sampler_harness.npz")
    for name, slot in [("camera", None), ("scatter", 0), ("light", 1), ("mesh", 2), ("environment", 3), ("decisions", 4)]:
        groups = np.zeros_like(g["px"]) if slot is None else 1 + g["vertex"] * 5 + slot
        bits = renderer.sampler_groups(g["px"], g["py"], g["index"], groups, 300, 0x5EED)
        assert np.array_equal(bits, g[name]), name
    rng = np.random.default_rng(7)
    n = 1 << 16
    px, py = rng.integers(0, 1 << 20, n), rng.integers(0, 1 << 20, n)
    for count in (1, 16, 64, 1000, 1 << 20):
        idx, grp = rng.integers(0, count, n), rng.integers(0, 5000, n)
        a = renderer.sampler_groups(px, py, idx, grp, count, 12345)
        b = oracle.sampler_bits(px, py, idx, grp, count, 12345, 1)
        assert np.array_equal(a, b), count


def test_brdf_atlas_matches_known_texels_and_oracle(renderer, oracle):
    lut = renderer.brdf_lut()
    k = json.loads((GOLDEN / "reference_kats.json").read_text())
    for x, y, e in k["brdf_texels"]:
        assert abs(lut[y, x, 0] - e) < k["brdf_tolerance"], (x, y, lut[y, x], e)
    ref = oracle.brdf_lut(False)
    # fp16 storage: agree to a couple of half ulps (2^-10 relative) plus an absolute floor.
    assert np.all(np.abs(lut - ref) <= 2e-3 * np.abs(ref) + 2e-4), float(np.abs(lut - ref).max())


def test_morton_codes_bit_exact(renderer, oracle, small_scene):
    o = oracle.OracleScene(small_scene)
    with renderer.install(small_scene) as s:
        assert np.array_equal(s.tlas_morton(), o.tlas_morton())
        for m in range(len(small_scene.meshes)):
            assert np.array_equal(s.blas_morton(m), o.blas_morton(m)), m


def test_primary_ids_match_oracle(renderer, oracle, small_scene):
    o = oracle.OracleScene(small_scene)
    prof = Profile.reference_transport(4, 16)
    rays = o.camera_rays(prof.c(), index=0)
    t_ref, ids_ref, _ = o.trace(rays, fp64=True)
    with renderer.install(small_scene) as s:
        t, ids, _ = s.trace(rays)
        mismatch = np.any(ids != ids_ref, axis=1)
        assert mismatch.mean() <= 1e-4, int(mismatch.sum())
        hit = ids_ref[:, 0] != 0xFFFFFFFF
        assert np.allclose(t[hit & ~mismatch], t_ref[hit & ~mismatch], rtol=1e-4, atol=1e-5)
        # The render's own first-sample IDs (camera rays built on the device).
        res = s.render(Profile.reference_transport(4, 16, sample_count=1), ids=True)
        pid = res.primary_ids.reshape(-1, 2)
        assert np.mean(np.any(pid != ids_ref, axis=1)) <= 1e-3
        assert res.stats["traversal_overflows"] == 0


def test_random_rays_closest_and_any_hits(renderer, oracle, small_scene):
    o = oracle.OracleScene(small_scene)
    rng = np.random.default_rng(11)
    n = 20000
    org = rng.uniform(-2, 12, (n, 3))
    d = rng.normal(size=(n, 3)); d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([org, d, np.full((n, 1), 1e30)], 1).astype(np.float32)
    t_ref, ids_ref, _ = o.trace(rays, fp64=True)
    # Shadow rays: finite reach, the any-hit traversal (first hit ends the walk, no
    # back-face culling: path.slang:630-684) against the oracle's any-hit query.
    reach = rays.copy()
    reach[:, 6] = rng.uniform(0.2, 12.0, n).astype(np.float32)
    _, any_ref, _ = o.trace(reach, fp64=True, any_hit=True)
    occ_ref = any_ref[:, 0] != 0xFFFFFFFF
    with renderer.install(small_scene) as s:
        t, ids, _ = s.trace(rays)
        occ = s.occluded(reach)
        # From inside a sphere every direction is occluded (back faces count for shadows)
        # while the closest-hit query culls them.
        inside = np.concatenate([np.tile(small_scene.instance_rows[0, :, 3], (64, 1)), d[:64], np.full((64, 1), 1e30)], 1)
        occ_inside = s.occluded(inside.astype(np.float32))
        _, ids_inside, _ = s.trace(inside.astype(np.float32))
    mismatch = np.any(ids != ids_ref, axis=1)
    assert mismatch.mean() <= 2e-3, int(mismatch.sum())
    assert 0.2 < occ_ref.mean() < 0.8, float(occ_ref.mean())       # a real mix of blocked and free rays
    assert np.mean(occ != occ_ref) <= 2e-3, int(np.sum(occ != occ_ref))
    assert occ_inside.all() and np.all(ids_inside[:, 0] != 0), ids_inside[:4]


def _small_profile(spp=16, **kw):
    return Profile.reference_transport(4, spp, **kw)


def test_render_matches_fp64_oracle(renderer, oracle, small_scene):
    # Same sampler bits per sample: per-pixel agreement on most pixels, and the image
    # mean within 1% of the FP64 restatement.
    o = oracle.OracleScene(small_scene)
    prof = _small_profile(16)
    x0, y0, w, h = 96, 96, 64, 64
    ref, st_ref = o.render(prof.c(), x0, y0, w, h, fp64=True)
    with renderer.install(small_scene) as s:
        res = s.render(prof)
    img = res.image[y0:y0 + h, x0:x0 + w]
    assert np.isfinite(res.image).all() and res.stats["dropped_path_samples"] == 0
    m_gpu, m_ref = img[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
    assert np.all(np.abs(m_gpu / m_ref - 1) < 0.01), (m_gpu, m_ref)
    rel = np.abs(img[..., :3] - ref[..., :3]).sum(-1) / (ref[..., :3].sum(-1) + 1e-3)
    assert np.mean(rel < 1e-3) > 0.8, float(np.mean(rel < 1e-3))
    assert res.stats["traversal_overflows"] == 0


def test_full_image_matches_fp32_oracle_at_low_spp(renderer, oracle, small_scene):
    o = oracle.OracleScene(small_scene)
    prof = _small_profile(16, sample_count=2)
    ref, _ = o.render(prof.c(), fp64=False)
    with renderer.install(small_scene) as s:
        img = s.render(prof).image
    m_gpu, m_ref = img[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
    assert np.all(np.abs(m_gpu / m_ref - 1) < 0.01), (m_gpu, m_ref)
    rel = np.abs(img[..., :3] - ref[..., :3]).sum(-1) / (ref[..., :3].sum(-1) + 1e-3)
    assert np.mean(rel < 1e-3) > 0.8


def _per_pixel(img, ref):
    return np.abs(img[..., :3] - ref[..., :3]).sum(-1) / (ref[..., :3].sum(-1) + 1e-3)


def test_single_samples_match_fp32_oracle_on_the_device_atlas(renderer, oracle, small_scene):
    # One sample per pixel, the oracle reading the device-baked atlas: what is left is
    # the transport itself.  A sample either agrees to float rounding or its path took
    # another branch (a different triangle at a shared edge, a roulette or lobe choice
    # on the other side of its threshold after rounding) and differs entirely; those
    # branch flips are rare, and a 16-spp pixel differs once any of its samples flipped.
    o = oracle.OracleScene(small_scene, fp32=True, fp64=False)
    lut = renderer.brdf_lut()
    fracs = []
    with renderer.install(small_scene) as s:
        for k in range(4):
            prof = _small_profile(16, first_sample=k, sample_count=1)
            img = s.render(prof).image
            with oracle.atlas(lut):
                ref, _ = o.render(prof.c(), fp64=False)
            rel = _per_pixel(img, ref)
            fracs.append((float(np.mean(rel < 1e-4)), float(np.mean(rel > 1e-2))))
    print("single samples vs FP32 oracle (device atlas): fraction within 1e-4, fraction beyond 1e-2:", fracs)
    for close, far in fracs:
        assert close > 0.97 and far < 0.02, fracs


@pytest.mark.parametrize("clamps", [(0.0, 10.0), (2.0, 0.5)])
def test_clamped_render_matches_oracle(renderer, oracle, small_scene, clamps):
    # sample_clamp.slang:1-25: the direct and indirect clamps of the production profile
    # (clamp_indirect = 10, constants.rs:262) and a tighter pair that bites often.
    o = oracle.OracleScene(small_scene, fp32=True, fp64=False)
    base = _small_profile(16, sample_count=4)
    prof = dataclasses.replace(base, clamp_direct=clamps[0], clamp_indirect=clamps[1])
    lut = renderer.brdf_lut()
    with renderer.install(small_scene) as s:
        img = s.render(prof).image
        free = s.render(base).image
    with oracle.atlas(lut):
        ref, _ = o.render(prof.c(), fp64=False)
        ref_free, _ = o.render(base.c(), fp64=False)
    assert not np.array_equal(img, free)                 # the clamp changed some samples
    removed = ref_free[..., :3].mean() - ref[..., :3].mean()
    assert removed > 0
    m, mr = img[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
    assert np.all(np.abs(m / mr - 1) < 0.01), (m, mr)
    # The energy the clamp removes agrees too.
    assert abs((free[..., :3].mean() - img[..., :3].mean()) / removed - 1) < 0.05
    assert np.mean(_per_pixel(img, ref) < 1e-3) > 0.8


def test_production_profile_matches_oracle(renderer, oracle, small_scene):
    # std/path defaults (constants.rs:256-267): bounces 12/4/4/12, transparent 8,
    # indirect clamp 10, light threshold 0.01 (adaptive stopping has its own test).
    o = oracle.OracleScene(small_scene, fp32=True, fp64=False)
    prof = Profile(samples=16, sample_count=4)
    lut = renderer.brdf_lut()
    with renderer.install(small_scene) as s:
        img = s.render(prof).image
    with oracle.atlas(lut):
        ref, _ = o.render(prof.c(), fp64=False)
    m, mr = img[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
    assert np.all(np.abs(m / mr - 1) < 0.01), (m, mr)
    assert np.mean(_per_pixel(img, ref) < 1e-3) > 0.8


def test_white_diffuse_under_coloured_environment(renderer):
    # environment_tests.rs:117-160: a white Lambert surface under a constant
    # environment of (1, 0.75, 0.5) returns it, within 3% (here exactly).
    g = S.grid((200.0, 200.0), (2, 2))
    m = S.material((1, 1, 1), 0.5, 0.0)
    m.specular_weight = 0.0
    rows = S.rows_from(1.0, (0, 0, 0))[None]
    cam = S.look_at((0, 5, 0.001), (0, 0, 0), width=32, height=32, fov_y_degrees=30)
    sc = S.Scene([g], rows, np.zeros(1, np.uint32), np.zeros(1, np.uint32), [m], [], cam,
                 S.environment((1.0, 0.75, 0.5)))
    with renderer.install(sc) as s:
        img = s.render(Profile.reference_transport(64, 16)).image
    mean = img[..., :3].reshape(-1, 3).mean(0)
    assert np.allclose(mean, [1.0, 0.75, 0.5], rtol=1e-5), mean


def test_deterministic_across_waves_and_runs(renderer, small_scene):
    with renderer.install(small_scene) as s:
        a = s.render(_small_profile(8)).image
        b = s.render(_small_profile(8)).image
        c = s.render(_small_profile(8, wave_samples=1)).image
        d = s.render(_small_profile(8, wave_samples=3)).image
        assert np.array_equal(a, b) and np.array_equal(a, c) and np.array_equal(a, d)
        # Resume: samples [0,4) + [4,8) equal [0,8).
        h0 = s.render(_small_profile(8, first_sample=0, sample_count=4)).image
        h1 = s.render(_small_profile(8, first_sample=4, sample_count=4)).image
        assert np.allclose((h0 + h1) / 2, a, rtol=1e-5, atol=1e-6)


def test_overlapped_waves_equal_serial_waves(renderer, small_scene):
    # Waves of one render alternate between two streams and wavefronts; the accumulation
    # keeps wave order, so the image and the counts equal one wave after another.
    with renderer.install(small_scene) as s:
        a = s.render(_small_profile(8, wave_samples=1))
        b = s.render(_small_profile(8, wave_samples=1, flags=abi.PROFILE_SERIAL_WAVES))
    assert np.array_equal(a.image, b.image)
    for k in ("extension_rays", "shadow_rays", "dropped_path_samples", "dropped_light_samples", "traversal_overflows"):
        assert a.stats[k] == b.stats[k], k


def test_update_instances_equals_fresh_install(renderer, small_scene):
    moved = S.spheres_scene()
    moved.instance_rows = small_scene.instance_rows.copy()
    moved.instance_rows[:64, 1, 3] += 0.5
    with renderer.install(small_scene) as s:
        s.update_instances(moved.instance_rows)
        a = s.render(_small_profile(4)).image
    with renderer.install(moved) as s2:
        b = s2.render(_small_profile(4)).image
    assert np.array_equal(a, b)


def test_tiny_scenes_and_errors(renderer):
    tri = S.Mesh(np.array([[0, 0, 0], [1, 0, 0], [0, 0, -1]], np.float32), np.array([[0, 1, 0]] * 3, np.float32),
                 np.array([[0, 1, 2]], np.uint32))
    cam = S.look_at((0.3, 2, -0.3), (0.3, 0, -0.3), width=16, height=16, fov_y_degrees=20)
    light = S.area_light((0.3, 3, -0.3), (0, -1, 0), (1, 0, 0), 1, 1, 10.0)
    sc = S.Scene([tri], S.rows_from(1.0, (0, 0, 0))[None], np.zeros(1, np.uint32), np.zeros(1, np.uint32), [S.material()],
                 [light], cam, S.environment())
    with renderer.install(sc) as s:
        img = s.render(Profile.reference_transport(4, 4)).image
        assert np.isfinite(img).all() and img[..., :3].max() > 0
        with pytest.raises(abi.VkbError) as e:     # adaptive stopping needs the whole exposure
            s.render(Profile(samples=4, adaptive=True, first_sample=1))
        assert e.value.status == abi.VKB_UNSUPPORTED
        assert np.isfinite(s.render(Profile(samples=4, adaptive=True)).image).all()
        with pytest.raises(abi.VkbError):
            s.render(Profile(samples=4, first_sample=9))
    bad = S.Scene([tri], S.rows_from(1.0, (0, 0, 0))[None], np.array([3], np.uint32), np.zeros(1, np.uint32), [S.material()],
                  [], cam, S.environment())
    with pytest.raises(abi.VkbError) as e:
        renderer.install(bad)
    assert e.value.status == abi.VKB_INVALID_ARG
    # One and two instances under both TLAS builders; an unknown builder is refused.
    for builder in (abi.TLAS_LBVH, abi.TLAS_PLOC):
        for k in (1, 2):
            rows = np.stack([S.rows_from(1.0, (0.0, 0.0, 0.0)), S.rows_from(1.0, (0.5, 0.1, 0.0))])[:k]
            sk = S.Scene([tri], rows, np.zeros(k, np.uint32), np.zeros(k, np.uint32), [S.material()], [light], cam,
                         S.environment(), tlas_builder=builder)
            with renderer.install(sk) as s:
                assert s.tlas_stats()["valid"]
                assert np.isfinite(s.render(Profile.reference_transport(4, 2)).image).all()
    with pytest.raises(abi.VkbError) as e:
        renderer.install(S.Scene([tri], S.rows_from(1.0, (0, 0, 0))[None], np.zeros(1, np.uint32), np.zeros(1, np.uint32),
                                 [S.material()], [light], cam, S.environment(), tlas_builder=7))
    assert e.value.status == abi.VKB_INVALID_ARG


@pytest.mark.parametrize("builder", [abi.TLAS_LBVH, abi.TLAS_PLOC])
def test_tlas_refit_matches_rebuild_and_follows_the_quarter_rule(renderer, small_scene, builder):
    # rt.rs:1465-1476: refit until the changed object bytes reach a quarter of the object buffer.
    small_scene = dataclasses.replace(small_scene, tlas_builder=builder)
    rows = small_scene.instance_rows.copy()
    with renderer.install(small_scene) as s:
        base = s.info()
        few = rows.copy(); few[:8, 1, 3] += 0.05                  # 8 of 65 rows: below a quarter -> refit
        s.update_instances(few, policy=0)
        i1 = s.info()
        assert i1["tlas_refits"] == base["tlas_refits"] + 1 and i1["tlas_rebuilds"] == base["tlas_rebuilds"]
        refit_img = s.render(_small_profile(4)).image
        assert s.tlas_stats()["valid"]
        s.update_instances(few, policy=1)                         # same rows, forced rebuild
        rebuilt_img = s.render(_small_profile(4)).image
        assert np.array_equal(refit_img, rebuilt_img)
        more = few.copy(); more[8:25, 1, 3] += 0.05               # 17 rows since the forced rebuild: >= 1/4 -> rebuild
        s.update_instances(more, policy=0)
        i2 = s.info()
        assert i2["tlas_rebuilds"] == i1["tlas_rebuilds"] + 2 and i2["motion_bytes"] == 0
        s.update_instances(more, policy=0)                        # nothing changed: no work
        assert s.info()["tlas_refits"] == i2["tlas_refits"]
        big = more.copy(); big[:, 1, 3] += 0.3
        s.update_instances(big, policy=2)                         # forced refit after large motion
        a = s.render(_small_profile(4)).image
        s.update_instances(big, policy=1)
        b = s.render(_small_profile(4)).image
        assert np.array_equal(a, b)


def _crowd_scene(seed=5):
    """20,000 instances of a 500-triangle sphere: 4,000 coincident at one spot, 6,000 in
    a dense clump, the rest scattered -- equal merge costs and near-equal Morton codes
    for the TLAS builder."""
    rng = np.random.default_rng(seed)
    mesh = S.geodesic_sphere(5)
    centers = np.concatenate([np.tile([[5.0, 5.0, 5.0]], (4000, 1)), rng.normal(5.0, 0.3, (6000, 3)),
                              rng.uniform(0.0, 10.0, (10000, 3))])
    radii = np.concatenate([np.full(4000, 0.4), rng.uniform(0.02, 0.1, 16000)])
    rows = np.stack([S.rows_from(float(r), tuple(c)) for r, c in zip(radii, centers)]).astype(np.float32)
    cam = S.look_at(eye=(5.0, 5.0, -12.0), target=(5.0, 5.0, 5.0), width=96, height=96)
    return S.Scene([mesh], rows, np.zeros(len(rows), np.uint32), np.zeros(len(rows), np.uint32), [S.material()],
                   [S.sun_light((0.3, -1.0, 0.2))], cam, S.environment((0.2, 0.2, 0.2)), name="crowd")


@pytest.mark.parametrize("builder", [abi.TLAS_LBVH, abi.TLAS_PLOC])
def test_tlas_over_coincident_and_clustered_instances(renderer, oracle, builder):
    # Coincident instances tie on t, so which instance is reported may differ; the hit
    # distance and hit/miss must not.
    sc = _crowd_scene()
    sc.tlas_builder = builder
    o = oracle.OracleScene(sc, fp64=False)
    rng = np.random.default_rng(3)
    n = 20000
    org = rng.uniform(-2, 12, (n, 3))
    d = rng.normal(size=(n, 3)); d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([org, d, np.full((n, 1), 1e30)], 1).astype(np.float32)
    t_ref, ids_ref, _ = o.trace(rays, fp64=False)
    with renderer.install(sc) as s:
        t, ids, _ = s.trace(rays)
        st = s.tlas_stats()
        assert st["valid"] and st["max_depth"] < 200 and np.isfinite(st["sah_cost"]), st
    hit, hit_ref = ids[:, 0] != 0xffffffff, ids_ref[:, 0] != 0xffffffff
    assert np.mean(hit != hit_ref) <= 1e-3
    both = hit & hit_ref
    assert both.sum() > 1000
    rel = np.abs(t[both] - t_ref[both]) / np.maximum(t_ref[both], 1e-3)
    assert np.mean(rel > 1e-4) <= 2e-3


def test_adaptive_stopping_matches_the_oracle(renderer, oracle):
    # path.slang:1792-1837: per-sample stopping with the 3x3 rule, whole image; the GPU
    # (one sample per wave) and the FP32 oracle (sample-major) take the same decisions up
    # to float differences in the moments, so the traced work and the image agree closely.
    sc = S.spheres_scene(width=96, height=96)
    prof = Profile.reference_transport(4, 64, adaptive=True, adaptive_threshold=0.05)
    o = oracle.OracleScene(sc, fp32=True, fp64=False)
    ref, st_ref = o.render(prof.c(), fp64=False)
    with renderer.install(sc) as s:
        res = s.render(prof)
        plain = s.render(Profile.reference_transport(4, 64))
        again = s.render(prof)
    assert np.array_equal(res.image, again.image)
    st = res.stats
    assert st["samples_skipped"] > 0.05 * 96 * 96 * 64
    assert abs(st["extension_rays"] / st_ref["extension_rays"] - 1) < 0.02
    assert st["extension_rays"] < plain.stats["extension_rays"]
    m, mr = res.image[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
    assert np.all(np.abs(m / mr - 1) < 0.01), (m, mr)
    with pytest.raises(abi.VkbError) as e:
        s2 = renderer.install(sc)
        try:
            s2.render(Profile.reference_transport(4, 64, adaptive=True, first_sample=8))
        finally:
            s2.close()
    assert e.value.status == abi.VKB_UNSUPPORTED
