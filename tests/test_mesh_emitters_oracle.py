"""The oracle's emissive meshes (emitters.rs:22-44, emitter_weights.slang,
emitter_mesh_proposal.slang, path.slang:996-1002,1121-1167,1580-1591) on CPU: the weight
tree holds world area x emission power with mean inner nodes; triangle probabilities are
the half-and-half mix of that tree and the uniform choice and sum to one; sampling draws
triangles at those probabilities, uniformly over each triangle; a white Lambert plane under
a lamp returns the lamp's form factor x its radiance; a lamp seen directly returns its
radiance."""
import numpy as np
import pytest

from vork_b200 import Profile, scene as S

LUM = np.array([0.2126, 0.7152, 0.0722], np.float32)


def _source_triangles(sc):
    """(instance, primitive, world area, power) of every source triangle in source order."""
    out = []
    for i, (m, k) in enumerate(zip(sc.instance_mesh, sc.instance_material)):
        mat = sc.materials[k]
        col = np.array(mat.emission_color[:], np.float32)
        if not (mat.emission_luminance > 0 and np.any(col != 0)):
            continue
        mesh = sc.meshes[m]
        M = sc.instance_rows[i][:, :3].astype(np.float64)
        p = mesh.positions[mesh.indices].astype(np.float64)       # (T,3,3)
        a = (p[:, 1] - p[:, 0]) @ M.T
        b = (p[:, 2] - p[:, 0]) @ M.T
        area = 0.5 * np.linalg.norm(np.cross(a, b), axis=1)
        power = float(np.dot(np.maximum(col, 0), LUM)) * max(mat.emission_luminance, 0.0)
        for t in range(len(area)):
            out.append((i, t, area[t], power))
    return out


def test_weight_tree_and_probabilities(oracle):
    sc = S.lamp_scene(lamps=3, spheres=2)
    o = oracle.OracleScene(sc)
    src = _source_triangles(sc)
    tree, leaves = o.mesh_tree()
    n = len(src)
    assert o.mesh_triangles() == n and leaves == 1 << (n - 1).bit_length()
    w = np.array([a * p for _, _, a, p in src])
    assert np.allclose(tree[leaves:leaves + n], w, rtol=2e-5)
    assert np.all(tree[leaves + n:] == 0)
    inner = np.arange(1, leaves)
    assert np.array_equal(tree[inner], np.float32(0.5) * tree[2 * inner] + np.float32(0.5) * tree[2 * inner + 1])
    inst = np.array([s[0] for s in src], np.uint32)
    prim = np.array([s[1] for s in src], np.uint32)
    prob = o.mesh_probability(inst, prim)
    assert abs(prob.astype(np.float64).sum() - 1) < 1e-5
    assert np.allclose(prob, 0.5 * w / w.sum() + 0.5 / n, rtol=1e-4)
    # Triangles that are not sources have no probability.
    assert np.all(o.mesh_probability(np.zeros(4, np.uint32), np.arange(4, dtype=np.uint32)) == 0)


def test_sampling_follows_the_probabilities(oracle):
    sc = S.lamp_scene(lamps=3, spheres=2)
    o = oracle.OracleScene(sc)
    src = _source_triangles(sc)
    n = len(src)
    index = {(s[0], s[1]): k for k, s in enumerate(src)}
    u = np.random.default_rng(3).random((400000, 3)).astype(np.float32)
    inst, prim, b, pr = o.mesh_sample(u)
    k = np.array([index[(int(a), int(c))] for a, c in zip(inst, prim)])
    counts = np.bincount(k, minlength=n)
    expected = o.mesh_probability(np.array([s[0] for s in src], np.uint32), np.array([s[1] for s in src], np.uint32)) * len(u)
    # Every sample reports the probability of the triangle it drew.
    assert np.allclose(pr, o.mesh_probability(inst, prim))
    big = expected > 200
    z = (counts[big] - expected[big]) / np.sqrt(expected[big])
    assert np.abs(z).max() < 5, np.abs(z).max()
    chi2 = float(((counts - expected) ** 2 / expected).sum())
    assert chi2 < n + 6 * np.sqrt(2 * n), (chi2, n)
    # Uniform over each triangle: barycentrics inside, centroid mean.
    assert np.all(b >= 0) and np.all(b.sum(1) <= 1 + 1e-6)
    assert np.allclose(b.mean(0), 1 / 3, atol=3e-3)


def _corner(a, b):
    """Form factor from a point to an a x b rectangle in a parallel plane at unit height,
    the point below one corner (signed in a and b)."""
    sa, sb = np.sqrt(1 + a * a), np.sqrt(1 + b * b)
    return (a / sa * np.arctan(b / sa) + b / sb * np.arctan(a / sb)) / (2 * np.pi)


def _lamp_over_plane(width=8, height=8, double_sided=False, lamp=(1.2, 0.8), h=1.0, luminance=10.0):
    g = S.grid((200.0, 200.0), (2, 2))
    white = S.material((1, 1, 1), 0.5, 0.0)
    white.specular_weight = 0.0
    q = S.grid((1.0, 1.0), (1, 1))
    r = np.zeros((3, 4), np.float32)
    r[0, 0], r[1, 1], r[2, 2] = lamp[0], -1.0, -lamp[1]
    r[:, 3] = (0.0, h, 0.0)
    cam = S.look_at((0, 5, 0.001), (0, 0, 0), width=width, height=height, fov_y_degrees=2)
    rows = np.stack([S.rows_from(1.0, (0, 0, 0)), r]).astype(np.float32)
    return S.Scene([g, q], rows, np.array([0, 1], np.uint32), np.array([0, 1], np.uint32),
                   [white, S.emissive((1.0, 0.8, 0.6), luminance, double_sided)], [], cam, S.environment((0.0, 0.0, 0.0)))


def lamp_form_factor(lamp=(1.2, 0.8), h=1.0, half_view=5 * np.tan(np.radians(1.0))):
    """Mean form factor of the lamp over the plane patch the 2-degree camera sees."""
    xs = np.linspace(-half_view, half_view, 41)
    X, Z = np.meshgrid(xs, xs)
    x0, x1, z0, z1 = -lamp[0] / 2, lamp[0] / 2, -lamp[1] / 2, lamp[1] / 2
    F = (_corner((x1 - X) / h, (z1 - Z) / h) - _corner((x0 - X) / h, (z1 - Z) / h)
         - _corner((x1 - X) / h, (z0 - Z) / h) + _corner((x0 - X) / h, (z0 - Z) / h))
    return float(F.mean())


def test_white_plane_under_a_lamp_returns_its_form_factor(oracle):
    # Mesh NEE plus MIS-weighted emitter hits of BSDF samples: an unbiased estimate of the
    # plane's outgoing radiance, albedo 1 x radiance x form factor.
    sc = _lamp_over_plane()
    o = oracle.OracleScene(sc)
    img, st = o.render(Profile.reference_transport(2, 256).c(), fp64=True)
    expected = lamp_form_factor() * 10.0 * np.array([1.0, 0.8, 0.6])
    got = img[..., :3].mean((0, 1))
    assert np.allclose(got, expected, rtol=5e-3), (got, expected)
    assert st["shadow_rays"] > 0


def test_lamp_seen_directly_returns_its_radiance(oracle):
    sc = _lamp_over_plane(double_sided=True)
    sc.camera = S.look_at((0, 3, 0.001), (0, 1, 0), width=8, height=8, fov_y_degrees=10)
    o = oracle.OracleScene(sc)
    img, _ = o.render(Profile.reference_transport(2, 4).c(), fp64=True)
    assert np.allclose(img[..., :3], np.array([1.0, 0.8, 0.6]) * 10.0, rtol=1e-6)


def test_single_sided_lamp_is_dark_from_behind(oracle):
    # The lamp faces down: a camera below sees its emitting side, one above sees through it.
    sc = _lamp_over_plane()
    sc.camera = S.look_at((0, 0.2, 0.001), (0, 1, 0), width=8, height=8, fov_y_degrees=10)
    below, _ = oracle.OracleScene(sc).render(Profile.reference_transport(2, 2).c(), fp64=True)
    assert np.allclose(below[..., :3], np.array([1.0, 0.8, 0.6]) * 10.0, rtol=1e-6)
    sc.camera = S.look_at((0, 3, 0.001), (0, 1, 0), width=8, height=8, fov_y_degrees=10)
    above, _ = oracle.OracleScene(sc).render(Profile.reference_transport(2, 2).c(), fp64=True)
    # The floor under the lamp (radiance x form factor, 0.23 x radiance here), not the lamp.
    assert np.all(above[..., :3] < 0.5 * np.array([1.0, 0.8, 0.6]) * 10.0) and np.all(above[..., :3] > 0)


@pytest.mark.parametrize("fp64", [False, True])
def test_lamp_scene_renders_finite_in_both_precisions(oracle, fp64):
    sc = S.lamp_scene(width=24, height=16, lamps=2, spheres=3)
    img, st = oracle.OracleScene(sc).render(Profile.reference_transport(4, 8).c(), fp64=fp64)
    assert np.all(np.isfinite(img)) and img[..., :3].mean() > 0.01 and st["dropped_path_samples"] == 0
