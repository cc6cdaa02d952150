"""The oracle against the reference's own known answers and invariants (CPU only).

Each test names the reference test it restates.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def kats():
    return json.loads((GOLDEN / "reference_kats.json").read_text())


def test_sobol_directions_match_published_table(oracle):
    # path_sampler.rs:81-93 sobol_table_matches_published_direction_numbers
    d = oracle.sobol_directions()
    k = kats()
    assert d[2][:8].tolist() == k["sobol_dim4_directions"]
    assert (oracle.sobol_points(8) >> 29).tolist() == k["sobol_first_points_eighths"]


def test_table_and_recurrence_samplers_agree(oracle):
    # The shader's generator recurrences (path_sampler.slang:80-88) against the table form.
    rng = np.random.default_rng(1)
    n = 4000
    px, py = rng.integers(0, 1 << 16, n), rng.integers(0, 1 << 16, n)
    for count in (1, 2, 16, 300, 1024, 4096):
        idx = rng.integers(0, count, n)
        g = rng.integers(0, 200, n)
        a = oracle.sampler_bits(px, py, idx, g, count, 0x5EED, 0)
        b = oracle.sampler_bits(px, py, idx, g, count, 0x5EED, 1)
        assert np.array_equal(a, b), count


def test_sampler_matches_golden_harness(oracle):
    # The reference GPU-parity harness (path_sampler.rs:266-276) as golden vectors.
    g = np.load(GOLDEN / "sampler_harness.npz")
    for name, slot in [("camera", None), ("scatter", 0), ("light", 1), ("mesh", 2), ("environment", 3), ("decisions", 4)]:
        groups = np.zeros_like(g["px"]) if slot is None else 1 + g["vertex"] * 5 + slot
        bits = oracle.sampler_bits(g["px"], g["py"], g["index"], groups, 300, 0x5EED, 0)
        assert np.array_equal(bits, g[name]), name


@pytest.mark.parametrize("pixel,stream,groups", [((0, 0), 0, range(0, 3)), ((913, 77), 0x5EED, range(5, 7)),
                                                 ((0xFFFFFFFF, 3), 1, range(40, 41))])
def test_every_power_of_two_prefix_is_a_net(oracle, pixel, stream, groups):
    # path_sampler.rs:99-133
    pairs = [(0, 1, 0), (0, 2, 1), (0, 3, 2), (1, 2, 1), (1, 3, 2), (2, 3, 1)]
    for g in groups:
        for count in (1, 2, 4, 16, 64, 256, 1024):
            idx = np.arange(count)
            pts = oracle.sampler_bits(np.full(count, pixel[0]), np.full(count, pixel[1]), idx, np.full(count, g), count, stream, 0)
            k = int(math.log2(count))
            for c in range(4):
                cells = (pts[:, c] >> (32 - k)) if k else np.zeros(count, np.uint32)
                assert len(np.unique(cells)) == count
            for a, b, t in pairs:
                if k < t:
                    continue
                for split in range(k - t + 1):
                    ka, kb = split, k - t - split
                    ca = (pts[:, a] >> (32 - ka)) if ka else np.zeros(count, np.uint32)
                    cb = (pts[:, b] >> (32 - kb)) if kb else np.zeros(count, np.uint32)
                    hits = np.bincount((ca.astype(np.int64) << kb) | cb, minlength=1 << (ka + kb))
                    assert np.all(hits == (1 << t))


def test_groups_and_pixels_are_decorrelated(oracle):
    # path_sampler.rs:137-174 (pooled correlations at Monte Carlo size)
    count, pixels = 64, 256
    p = np.repeat(np.arange(pixels), count)
    i = np.tile(np.arange(count), pixels)
    unit = lambda b: ((b >> 9).astype(np.float64) + 0.5) / 8388608.0
    bound = 5.0 / math.sqrt(pixels * count)
    for ga, gb in [(0, 1), (1, 2), (1, 5), (2, 6), (17, 400)]:
        xa = unit(oracle.sampler_bits(p, 3 * p + 1, i, np.full_like(p, ga), count, 7, 0)) - 0.5
        xb = unit(oracle.sampler_bits(p, 3 * p + 1, i, np.full_like(p, gb), count, 7, 0)) - 0.5
        for a in range(4):
            for b in range(4):
                r = float((xa[:, a] * xb[:, b]).mean() * 12.0)
                assert abs(r) < bound, (ga, gb, a, b, r)


def test_film_table_matches_blackman_harris_cdf(oracle):
    # sampling.rs:281-300 path_filter_lookup_matches_blackman_harris_cdf
    t = oracle.filter_table().astype(np.float64)
    n = 1024
    assert t[0] == -1.5 and t[n] == 1.5
    assert np.all(np.diff(t) >= 0)
    assert np.all(np.abs(t + t[::-1]) < 1e-6)
    cdf = oracle.lib().oracle_filter_cdf
    for i in range(n):
        for f in (0.0, 0.25, 0.5, 0.75):
            x = t[i] * (1 - f) + t[i + 1] * f
            assert abs(cdf(x) - (i + f) / n) < 0.0007  # the reference's bound


@pytest.mark.parametrize("fp64", [False, True])
def test_brdf_atlas_known_texels(oracle, fp64):
    # environment/brdf_tests.rs:97-104 (+ every dielectric texel written, alpha 1 or 0)
    lut = oracle.brdf_lut(fp64)
    k = kats()
    for x, y, e in k["brdf_texels"]:
        assert abs(lut[y, x, 0] - e) < k["brdf_tolerance"], (x, y, lut[y, x], e)
        assert lut[y, x, 1] == 0 and lut[y, x, 2] == 0
    assert np.isfinite(lut).all()
    ys, xs = np.mgrid[128:2240, 0:128]
    valid = ((ys - 128) // 64) * 2 + xs // 64 <= 64
    assert np.array_equal(lut[128:, :, 3], valid.astype(np.float32))
    # Moments: unit-Fresnel directional albedo <= 1; E_avg only in column 0.
    m = lut[:128, :, 0] + lut[:128, :, 1]
    assert m.max() <= 1.0005 and m.min() > 0
    assert np.all(lut[:128, 1:, 3] == 0) and np.all(lut[:128, 0, 3] > 0)


def _light(kind):
    from vork_b200 import abi
    l = abi.VkbLight()
    l.position[:] = [0, 0, 4, 1]
    l.direction[:] = [0, 0, -1, -1]
    l.radiance[:] = [1, 1, 1, 1]
    l.emitter_u[:] = [4, 0, 0, 0]
    l.emitter_v[:] = [0, 2, 0, 0]
    if kind in (1, 4):
        l.position[3] = 0
    if kind in (2, 3):
        l.params[1] = 2
    if kind == 3:
        l.position[3] = 2
    if kind == 4:
        l.params[1] = 0.4
    if kind >= 5:
        l.position[3] = 3
        l.emitter_u[3] = 1 if kind == 6 else 0
    return l


def test_emitter_endpoints_and_conditional_pdfs(oracle):
    # light_connection_tests.rs:8-84 connection_shape_endpoints_and_conditional_pdfs
    rows = []
    for kind in range(7):
        l = _light(kind)
        ep_err = pdf_err = cosine = 0.0
        for y in range(32):
            for x in range(32):
                u = ((x + 0.5) / 32, (y + 0.5) / 32)
                d, rad, pdf, dist = oracle.emitter_sample(l, (0, 0, 0), u)
                endpoint = np.asarray(d) * dist
                cosine += d[2] / 1024
                if kind in (2, 3):
                    ep_err = max(ep_err, abs(np.linalg.norm(endpoint - np.array([0, 0, 4])) - 2))
                    pdf_err = max(pdf_err, abs(pdf / (1 / (2 * math.pi * (1 - math.sqrt(0.75)))) - 1))
                elif kind == 4:
                    pdf_err = max(pdf_err, abs(pdf * (2 * math.pi * (1 - math.cos(0.4))) - 1))
                elif kind >= 5:
                    ep_err = max(ep_err, abs(endpoint[2] - 4))
                    q = endpoint[:2] / np.array([2.0, 1.0])
                    ep_err = max(ep_err, max(float(q @ q) - 1, 0) if kind == 6 else max(max(abs(q[0]), abs(q[1])) - 1, 0))
                    area = 2 * math.pi if kind == 6 else 8
                    pdf_err = max(pdf_err, abs(pdf * area * d[2] / (dist * dist) - 1))
                else:
                    pdf_err = max(pdf_err, abs(pdf))
        rows.append((ep_err, pdf_err, cosine))
    for kind, r in enumerate(rows):
        assert r[0] < 1e-4 and r[1] < 1e-4, (kind, r)
    sphere_mean = (1 + math.sqrt(0.75)) * 0.5
    assert abs(rows[2][2] - sphere_mean) < 1e-5 and abs(rows[3][2] - sphere_mean) < 1e-5
    assert abs(rows[4][2] - (1 + math.cos(0.4)) * 0.5) < 1e-5


def test_area_light_radiance_is_energy_over_pi_area(oracle):
    # lights.rs:99-142 with emitter.slang:143: L = radiance / (pi * area)
    from vork_b200 import scene
    l = scene.area_light((0, 5, 0), (0, -1, 0), (1, 0, 0), 2.0, 3.0, radiance=20.0)
    rad, pdf, dist = oracle.emitter_eval(l, (0.1, 0, 0.2), (0, 1, 0))
    assert np.allclose(rad, 20.0, rtol=1e-6) and abs(dist - 5.0) < 1e-9
    assert abs(pdf - 25.0 / 6.0) < 1e-9


def test_bsdf_sample_weight_is_eval_over_pdf_and_diffuse_white_is_one(oracle):
    # bsdf.slang:446-511: a white Lambert surface with no specular returns weight 1.
    from vork_b200 import scene
    m = scene.material((1, 1, 1), 0.5, 0.0)
    m.specular_weight = 0.0
    rng = np.random.default_rng(0)
    for _ in range(200):
        v = rng.normal(size=3); v[2] = abs(v[2]) + 0.05; v /= np.linalg.norm(v)
        d, w, pdf, ev = oracle.bsdf_sample(m, v, rng.random(3))
        assert ev == 4 and pdf > 0 and np.allclose(w, 1.0, atol=1e-12)


def test_metal_sampling_preserves_energy_bound(oracle):
    # GGX + F82 with Kulla-Conty compensation: the mean weight of a white-ish metal stays <= 1.02.
    from vork_b200 import scene
    rng = np.random.default_rng(2)
    for rough in (0.05, 0.3, 0.7, 1.0):
        m = scene.material((0.95, 0.95, 0.95), rough, 1.0)
        v = np.array([0.3, 0.0, 0.954]); v /= np.linalg.norm(v)
        ws = []
        for _ in range(4000):
            d, w, pdf, ev = oracle.bsdf_sample(m, v, rng.random(3))
            ws.append(w[0] if ev else 0.0)
        assert np.mean(ws) <= 1.02, (rough, np.mean(ws))
        assert np.mean(ws) >= 0.85, (rough, np.mean(ws))


def test_guide_planes_of_the_oracle(oracle):
    # path.slang:1549-1571 restated: a white-world response of a specular-free Lambert
    # plane is its base colour, its normal the plane's; misses add zero coverage.
    import numpy as np
    from vork_b200 import Profile, scene as S
    g = S.grid((200.0, 200.0), (2, 2))
    m = S.material((0.8, 0.6, 0.4), 0.5, 0.0)
    m.specular_weight = 0.0
    cam = S.look_at((0, 5, 0.001), (0, 0, 0), width=8, height=8, fov_y_degrees=30)
    sc = S.Scene([g], S.rows_from(1.0, (0, 0, 0))[None], np.zeros(1, np.uint32), np.zeros(1, np.uint32), [m], [], cam,
                 S.environment((1.0, 0.75, 0.5)))
    o = oracle.OracleScene(sc)
    _, _, gd = o.render(Profile.reference_transport(4, 4).c(), fp64=True, guides=True)
    assert np.allclose(gd[:, :, 0].reshape(-1, 4), [0.8, 0.6, 0.4, 1.0], atol=1e-12)
    assert np.allclose(gd[:, :, 1].reshape(-1, 4), [0.0, 1.0, 0.0, 0.0], atol=1e-12)
    # A general scene: albedo in [0, 1], coverage the fraction of hits, unit-or-shorter normals.
    sc2 = S.spheres_scene(width=48, height=48)
    _, _, g2 = oracle.OracleScene(sc2, fp64=False).render(Profile.reference_transport(4, 4).c(), fp64=False, guides=True)
    a, n = g2[:, :, 0], g2[:, :, 1]
    assert np.all((a[..., :3] >= 0) & (a[..., :3] <= 1)) and np.all((a[..., 3] >= 0) & (a[..., 3] <= 1))
    assert 0.3 < a[..., 3].mean() < 1.0
    assert np.all(np.linalg.norm(n[..., :3], axis=-1) <= 1 + 1e-6) and np.all(n[..., 3] == 0)
