"""The plain method's large configuration against the oracle, through the C ABI.

The frame the headline benchmark renders: 1,000,000 boid-placed instances of a
500-triangle geodesic mesh, a 2M-triangle noise-displaced terrain, sun + constant sky,
1920x1080, depth 8.  The GPU renders the whole frame (at 16 spp instead of 64); the
oracle checks crops of it (FP32 over five 64x64 crops, FP64 on the centre), the
primary-ray instance/triangle IDs of every pixel (FP64), the TLAS Morton codes of all
1,000,001 instances (bit-exact, including the bit-30 wide-box rule that sends the
terrain to its own side of the root), and the same after a flock step and a rebuild.
"""
import dataclasses

import numpy as np
import pytest

from vork_b200 import Profile, scene as S

pytestmark = pytest.mark.gpu

DEPTH, SPP = 8, 16
CROPS = [(928, 508), (400, 200), (1456, 200), (400, 816), (1456, 816)]   # 64x64 crop corners
MISS = 0xFFFFFFFF


@pytest.fixture(scope="module")
def large(renderer, oracle):
    sc, flock = S.flock_scene()
    o = oracle.OracleScene(sc, fp32=True, fp64=True)
    s = renderer.install(sc)
    prof = Profile.reference_transport(DEPTH, SPP)
    res = s.render(prof, ids=True)
    yield sc, flock, o, s, res
    s.close()
    o.close()


def _crop(img, x0, y0, w=64, h=64):
    return img[y0:y0 + h, x0:x0 + w]


def test_large_frame_renders_cleanly(large):
    sc, _, _, _, res = large
    st = res.stats
    assert np.isfinite(res.image).all()
    assert st["traversal_overflows"] == 0 and st["dropped_path_samples"] == 0
    assert st["paths"] == 1920 * 1080 * SPP
    # The frame holds birds, terrain and sky: all three kinds of primary hit occur.
    inst = res.primary_ids[..., 0]
    n_birds = sc.instance_rows.shape[0] - 1
    assert np.mean(inst == MISS) > 0.01 and np.mean(inst == n_birds) > 0.05 and np.mean(inst < n_birds) > 0.01


def test_large_crops_match_fp32_oracle(large, renderer, oracle):
    # Same sampler bits per sample.  Crop means within 1%; per pixel, the oracle reading
    # the device-baked atlas isolates the transport from the fp16 atlas bake.
    _, _, o, _, res = large
    prof = Profile.reference_transport(DEPTH, SPP)
    lut = renderer.brdf_lut()
    close = []
    for x0, y0 in CROPS:
        with oracle.atlas(lut):
            ref, st = o.render(prof.c(), x0, y0, 64, 64, fp64=False)
        img = _crop(res.image, x0, y0)
        m, mr = img[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
        assert np.all(np.abs(m / mr - 1) < 0.01), ((x0, y0), m, mr)
        rel = np.abs(img[..., :3] - ref[..., :3]).sum(-1) / (ref[..., :3].sum(-1) + 1e-3)
        close.append(np.mean(rel < 1e-3))
    print("large-frame crops, fraction of pixels within 1e-3 of the FP32 oracle:", [round(float(c), 4) for c in close])
    assert min(close) > 0.8, close


def test_large_centre_crop_matches_fp64_oracle(large, oracle):
    _, _, o, _, res = large
    prof = Profile.reference_transport(DEPTH, SPP)
    x0, y0 = 944, 524
    ref, _ = o.render(prof.c(), x0, y0, 32, 32, fp64=True)
    img = _crop(res.image, x0, y0, 32, 32)
    m, mr = img[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
    print("large-frame centre crop vs FP64 oracle, mean ratio:", (m / mr).tolist())
    assert np.all(np.abs(m / mr - 1) < 0.01), (m, mr)


def test_large_primary_ids_match_fp64_oracle(large):
    # Every pixel's first camera ray, as the oracle builds it, traced by the GPU's
    # closest-hit traversal and by the FP64 oracle: IDs differ on at most 1e-4 of pixels,
    # and only where the two hits are the same surface point (a shared edge or vertex:
    # equal distance) or the ray grazes a silhouette.
    _, _, o, s, res = large
    prof = Profile.reference_transport(DEPTH, SPP)
    rays = o.camera_rays(prof.c(), index=0)
    t_ref, ids_ref, uv_ref = o.trace(rays, fp64=True)
    t, ids, uv = s.trace(rays)
    mismatch = np.any(ids != ids_ref, axis=1)
    print("large-frame primary IDs: mismatching pixels", int(mismatch.sum()), "of", len(ids))
    assert mismatch.mean() <= 1e-4, int(mismatch.sum())
    both = mismatch & (ids[:, 0] != MISS) & (ids_ref[:, 0] != MISS)
    assert np.all(np.abs(t[both] - t_ref[both]) <= 1e-4 * t_ref[both]), (t[both], t_ref[both])
    hit = ~mismatch & (ids_ref[:, 0] != MISS)
    assert np.allclose(t[hit], t_ref[hit], rtol=1e-4, atol=1e-5)
    # The render's own first-sample IDs (camera rays built on the device in fp32).
    pid = res.primary_ids.reshape(-1, 2)
    assert np.mean(np.any(pid != ids_ref, axis=1)) <= 1e-3


def test_large_tlas_morton_codes_bit_exact(large, oracle):
    sc, _, o, s, _ = large
    m, mr = s.tlas_morton(), o.tlas_morton()
    assert m.shape == (1_000_001,)
    assert np.array_equal(m, mr)
    # The terrain is wider than a quarter of the centroid spread: bit 30 sends it to its
    # own side of the root split; no bird is.
    assert (m[-1] >> 30) & 1 == 1 and not np.any((m[:-1] >> 30) & 1)
    st = s.tlas_stats()
    assert st["valid"], st


def test_large_flock_step_rebuild_matches_oracle(large, oracle):
    # One animation frame later (the benchmark's per-frame update): rebuilt TLAS, Morton
    # codes bit-exact on the new rows, and primary hits of a ray subset still agree.
    sc, flock, o, s, _ = large
    rows0 = sc.instance_rows.copy()
    flock.step()
    rows = np.concatenate([flock.rows(), sc.instance_rows[-1:]], 0).astype(np.float32)
    try:
        s.update_instances(rows, policy=0)          # every row moved: the quarter rule rebuilds
        info = s.info()
        assert info["tlas_rebuilds"] >= 2 and info["motion_bytes"] == 0
        moved = dataclasses.replace(sc, instance_rows=rows)
        om = oracle.OracleScene(moved, fp32=False, fp64=True)
        try:
            assert np.array_equal(s.tlas_morton(), om.tlas_morton())
            assert s.tlas_stats()["valid"]
            rays = om.camera_rays(Profile.reference_transport(DEPTH, SPP).c(), index=3)[::7]
            t_ref, ids_ref, _ = om.trace(rays, fp64=True)
            t, ids, _ = s.trace(rays)
            assert np.mean(np.any(ids != ids_ref, axis=1)) <= 1e-4
        finally:
            om.close()
    finally:
        s.update_instances(rows0, policy=1)
