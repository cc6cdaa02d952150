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
    # Same sampler bits per sample.  Most samples agree to float rounding; in this scene
    # of sub-pixel triangles about a tenth of them take another branch at a later bounce
    # (a secondary ray passing within an ulp of one of the millions of bird edges) and are
    # independent draws, so crop means carry that noise: all crops pooled within 1%, each
    # 64x64 crop within 2.5%.  The oracle reads the device-baked atlas.
    _, _, o, _, res = large
    prof = Profile.reference_transport(DEPTH, SPP)
    lut = renderer.brdf_lut()
    close, ratios, sums = [], [], np.zeros((2, 3))
    for x0, y0 in CROPS:
        with oracle.atlas(lut):
            ref, st = o.render(prof.c(), x0, y0, 64, 64, fp64=False)
        img = _crop(res.image, x0, y0)
        m, mr = img[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
        sums += [m, mr]
        ratios.append((m / mr).round(4).tolist())
        rel = np.abs(img[..., :3] - ref[..., :3]).sum(-1) / (ref[..., :3].sum(-1) + 1e-3)
        close.append(round(float(np.mean(rel < 1e-3)), 4))
    print("large-frame crops vs FP32 oracle: mean ratios", ratios, "pooled", (sums[0] / sums[1]).round(4).tolist(),
          "pixels within 1e-3", close)
    assert np.all(np.abs(sums[0] / sums[1] - 1) < 0.01), sums
    assert all(abs(r - 1) < 0.025 for rr in ratios for r in rr), ratios
    # Crops of open sky agree pixel for pixel; bird-dense crops only in the mean.
    assert max(close) == 1.0, close


def test_large_centre_crop_matches_fp64_oracle(large, oracle):
    _, _, o, _, res = large
    prof = Profile.reference_transport(DEPTH, SPP)
    x0, y0 = 928, 508
    ref, _ = o.render(prof.c(), x0, y0, 64, 64, fp64=True)
    img = _crop(res.image, x0, y0, 64, 64)
    m, mr = img[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
    print("large-frame centre crop vs FP64 oracle, mean ratio:", (m / mr).tolist())
    assert np.all(np.abs(m / mr - 1) < 0.01), (m, mr)


def _id_mismatches(ids, ids_ref, t, t_ref, uv, uv_ref):
    """(mismatching rays, of which unexplained).  A mismatch is explained when both hits lie
    at the same distance (a shared edge or vertex, or two instances passing through each
    other), or when the nearer hit -- the only one, if the other side missed -- lies within
    a few ulps of its triangle's edge (barycentric distance <= 2e-3 on triangles a few
    pixels wide): the rays 'within 1 ulp of a shared edge' of the parity requirement."""
    mismatch = np.any(ids != ids_ref, axis=1)
    hit, hit_ref = ids[:, 0] != MISS, ids_ref[:, 0] != MISS
    tie = hit & hit_ref & (np.abs(t - t_ref) <= 1e-4 * np.maximum(t_ref, 1e-3))
    edge = lambda w: np.minimum(np.minimum(w[:, 0], w[:, 1]), 1.0 - w[:, 0] - w[:, 1]) <= 2e-3
    gpu_near = hit & (~hit_ref | (t <= t_ref))
    near_edge = np.where(gpu_near, edge(uv), edge(uv_ref))
    return mismatch, mismatch & ~(tie | near_edge)


def test_large_primary_ids_match_fp64_oracle(large):
    # Every pixel's first camera ray, as the oracle builds it, traced by the GPU's
    # closest-hit traversal (watertight, fp32) and by the FP64 oracle (Moller-Trumbore):
    # IDs are equal except on rays at a shared edge (birds are ~2 pixels wide with 500
    # triangles each, so edges lie under many pixels); unexplained mismatches <= 1e-4.
    _, _, o, s, res = large
    prof = Profile.reference_transport(DEPTH, SPP)
    rays = o.camera_rays(prof.c(), index=0)
    t_ref, ids_ref, uv_ref = o.trace(rays, fp64=True)
    t, ids, uv = s.trace(rays)
    mismatch, unexplained = _id_mismatches(ids, ids_ref, t, t_ref, uv, uv_ref)
    print("large-frame primary IDs: mismatching pixels", int(mismatch.sum()), "unexplained", int(unexplained.sum()), "of", len(ids))
    assert unexplained.mean() <= 1e-4, int(unexplained.sum())
    assert mismatch.mean() <= 5e-4, int(mismatch.sum())
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
            t_ref, ids_ref, uv_ref = om.trace(rays, fp64=True)
            t, ids, uv = s.trace(rays)
            mismatch, unexplained = _id_mismatches(ids, ids_ref, t, t_ref, uv, uv_ref)
            assert unexplained.mean() <= 1e-4 and mismatch.mean() <= 5e-4, (int(mismatch.sum()), int(unexplained.sum()))
        finally:
            om.close()
    finally:
        s.update_instances(rows0, policy=1)
